// Contour surgery (contours.f90:350-683) on the GPU.
//
// The reference scans the nodes of each PV level in index order and mutates
// node positions and links as it goes, so later tests see earlier
// reconnections.  The B200 version keeps that exact semantics:
//   1. Box every segment of every level in parallel (the reference's
//      nbx = nint(1.2 sqrt(N_lev)) boxes, its bwxi/bwyi scaling and its
//      per-box list order, restored by sorting each box by node index).
//   2. Test every node against the segments of its box in parallel on the
//      unmodified state; nodes with a passing test are marked pending.
//   3. One warp per level replays the reference loop in node order, but only
//      at pending nodes.  A reconnection marks pending every later node whose
//      tests could read what it changed: the four modified nodes, their
//      original predecessors, and every node located in a box that lists a
//      segment starting at one of those.  All other nodes would find no
//      surgery in the reference either, so the result is identical.
//   4. The new contours are the cycles of the link array, each starting at
//      its lowest node index (the reference's avail() walk); they are found
//      by pointer jumping over runs of consecutive nodes, gathered into walk
//      order and renoded in parallel (renode.cu).
#include <math.h>
#include <stdio.h>

#include <algorithm>
#include <vector>

#include "renode.cuh"
#include "scan.cuh"
#include "state.cuh"

namespace casl {

struct LevelDesc {
  int ibeg, iend;   // node range (0-based, inclusive)
  int nbx, nby;
  int boxbase;      // first global box of the level
  int levt;         // indq value of the level
  double bwxi, bwyi;
};

struct SurgState {
  double *xq, *yq, *dx, *dy, *dsq;     // mutable
  int *nextq;                          // mutable
  const double *x0, *y0, *dx0, *dy0;   // original
  const int *nq0, *prev0, *lvl;
  const int *kb1, *bcnt, *bnode;       // segment lists per box
  const int *nb1, *nbcnt, *nbnode;     // nodes located per box
  unsigned char *pending;
};

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// Box range spanned by segment (i, i+dx) (contours.f90:467-480).
__device__ __forceinline__ void seg_boxes(double x, double y, double dx, double dy, const LevelDesc &L,
                                          const Consts &c, int &mbx1, int &mbx2, int &mby1,
                                          int &mby2) {
  double dnbx = (double)L.nbx, dnby = (double)L.nby;
  if (dx > 0.0) {
    mbx1 = f_int(dnbx + L.bwxi * (x - c.xmin));
    mbx2 = f_int(dnbx + L.bwxi * (x + dx - c.xmin));
  } else {
    mbx1 = f_int(dnbx + L.bwxi * (x + dx - c.xmin));
    mbx2 = f_int(dnbx + L.bwxi * (x - c.xmin));
  }
  if (dy > 0.0) {
    mby1 = f_int(dnby + L.bwyi * (y - c.ymin));
    mby2 = f_int(dnby + L.bwyi * (y + dy - c.ymin));
  } else {
    mby1 = f_int(dnby + L.bwyi * (y + dy - c.ymin));
    mby2 = f_int(dnby + L.bwyi * (y - c.ymin));
  }
  // a wrapped segment is shorter than half the domain; the clamps only guard
  // the device against corrupt input
  if (mbx2 - mbx1 + 1 > L.nbx) mbx2 = mbx1 + L.nbx - 1;
  if (mby2 - mby1 + 1 > L.nby) mby2 = mby1 + L.nby - 1;
  if (mbx2 < mbx1) mbx2 = mbx1;
  if (mby2 < mby1) mby2 = mby1;
}

__device__ __forceinline__ int node_box(double x, double y, const LevelDesc &L, const Consts &c) {
  int bx = clampi(f_int(L.bwxi * (x - c.xmin)), 0, L.nbx - 1);
  int by = clampi(f_int(L.bwyi * (y - c.ymin)), 0, L.nby - 1);
  return L.boxbase + L.nby * bx + by;
}

__global__ void k_sg_endnext(const int *__restrict__ i1q, const int *__restrict__ i2q, int nq,
                             int *__restrict__ endnext) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nq; j += gridDim.x * blockDim.x)
    endnext[i2q[j]] = i1q[j];
}

__global__ void k_sg_level_of(const LevelDesc *__restrict__ lev, int nlev, int npt,
                              int *__restrict__ lvl) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npt; i += gridDim.x * blockDim.x) {
    int lo = 0, hi = nlev - 1;
    while (lo < hi) {
      int mid = (lo + hi + 1) >> 1;
      if (lev[mid].ibeg <= i) lo = mid; else hi = mid - 1;
    }
    lvl[i] = lo;
  }
}

// work arrays dx, dy, dsq (contours.f90:397-415) and the original copies
__global__ void k_sg_init(const double *__restrict__ xq, const double *__restrict__ yq,
                          const int *__restrict__ nextq, const int *__restrict__ endnext, int npt,
                          double *dx, double *dy, double *dsq, double *x0, double *y0,
                          double *dx0, double *dy0, int *nq0, int *prev0, unsigned char *pending,
                          Consts c, int *err) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npt; i += gridDim.x * blockDim.x) {
    int a = endnext[i] >= 0 ? endnext[i] : i + 1;
    double xi = xq[i], yi = yq[i];
    if (!(xi >= c.xmin && xi < c.xmax && yi >= c.ymin && yi < c.ymax)) atomicExch(err, CASL_EDOMAIN);
    a = clampi(a, 0, npt - 1);
    double xx = xq[a] - xi;
    double ddx = xx - c.ellx * f_dint(xx * c.hlxi);
    double yy = yq[a] - yi;
    double ddy = yy - c.elly * f_dint(yy * c.hlyi);
    dx[i] = ddx; dy[i] = ddy; dsq[i] = ddx * ddx + ddy * ddy;
    dx0[i] = ddx; dy0[i] = ddy;
    x0[i] = xi; y0[i] = yi;
    int nx = nextq[i];
    if (nx < 0 || nx >= npt) { atomicExch(err, CASL_EINVAL); nx = i; }
    nq0[i] = nx;
    prev0[nx] = i;
    pending[i] = 0;
  }
}

__global__ void k_sg_count_entries(SurgState S, const LevelDesc *__restrict__ lev, int npt,
                                   int *__restrict__ ecount, int *__restrict__ nbox_of,
                                   int *__restrict__ nbcnt, Consts c) {
  for (int ib = blockIdx.x * blockDim.x + threadIdx.x; ib < npt; ib += gridDim.x * blockDim.x) {
    LevelDesc L = lev[S.lvl[ib]];
    int i = S.nq0[ib];
    int mbx1, mbx2, mby1, mby2;
    seg_boxes(S.x0[i], S.y0[i], S.dx0[i], S.dy0[i], L, c, mbx1, mbx2, mby1, mby2);
    ecount[ib] = (mbx2 - mbx1 + 1) * (mby2 - mby1 + 1);
    int nb = node_box(S.x0[i], S.y0[i], L, c);
    nbox_of[ib] = nb;
    atomicAdd(&nbcnt[nb], 1);
  }
}

__global__ void k_sg_emit(SurgState S, const LevelDesc *__restrict__ lev, int npt,
                          const int *__restrict__ eoff, int *__restrict__ ebox,
                          int *__restrict__ eib, int *__restrict__ bcnt, Consts c) {
  for (int ib = blockIdx.x * blockDim.x + threadIdx.x; ib < npt; ib += gridDim.x * blockDim.x) {
    LevelDesc L = lev[S.lvl[ib]];
    int i = S.nq0[ib];
    int mbx1, mbx2, mby1, mby2;
    seg_boxes(S.x0[i], S.y0[i], S.dx0[i], S.dy0[i], L, c, mbx1, mbx2, mby1, mby2);
    int e = eoff[ib];
    for (int mbx = mbx1; mbx <= mbx2; mbx++) {
      int mmbx = mbx % L.nbx;
      for (int mby = mby1; mby <= mby2; mby++) {
        int gb = L.boxbase + L.nby * mmbx + mby % L.nby;
        ebox[e] = gb;
        eib[e] = ib;
        e++;
        atomicAdd(&bcnt[gb], 1);
      }
    }
  }
}

__global__ void k_sg_place(const int *__restrict__ ebox, const int *__restrict__ eib, long long ne,
                           const int *__restrict__ kb1, int *__restrict__ cursor,
                           int *__restrict__ bnode) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < ne;
       e += (long long)gridDim.x * blockDim.x) {
    int gb = ebox[e];
    int pos = kb1[gb] + atomicAdd(&cursor[gb], 1);
    bnode[pos] = eib[e];
  }
}

__global__ void k_sg_place_nodes(const int *__restrict__ nbox_of, int npt,
                                 const int *__restrict__ nb1, int *__restrict__ cursor,
                                 int *__restrict__ nbnode) {
  for (int ib = blockIdx.x * blockDim.x + threadIdx.x; ib < npt; ib += gridDim.x * blockDim.x) {
    int gb = nbox_of[ib];
    nbnode[nb1[gb] + atomicAdd(&cursor[gb], 1)] = ib;
  }
}

// Restore the reference's per-box order (ascending node before the segment).
__global__ void k_sg_sort_boxes(const int *__restrict__ kb1, const int *__restrict__ bcnt,
                                int nbox, int *__restrict__ bnode) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nbox; b += gridDim.x * blockDim.x) {
    int s = kb1[b], n = bcnt[b];
    for (int a = 1; a < n; a++) {
      int v = bnode[s + a], k = a - 1;
      while (k >= 0 && bnode[s + k] > v) {
        bnode[s + k + 1] = bnode[s + k];
        k--;
      }
      bnode[s + k + 1] = v;
    }
  }
}

// The two tests of contours.f90:542-563.
__device__ __forceinline__ bool surg_test(double xi, double yi, double xs, double ys, double dxs,
                                          double dys, double dsqs, const Consts &c) {
  double xx = xs - xi;
  double delx = xx - c.ellx * f_dint(xx * c.hlxi);
  double yy = ys - yi;
  double dely = yy - c.elly * f_dint(yy * c.hlyi);
  double aa = delx * dxs + dely * dys;
  if (aa * (aa + dsqs) + c.d4small < 0.0) {
    double cr = delx * dys - dely * dxs;
    double cc = cr * cr;
    if (cc * (cc - c.dm2 * dsqs) < 0.0) return true;
  }
  return false;
}

// Parallel candidate detection on the unmodified state.
__global__ void k_sg_candidates(SurgState S, const LevelDesc *__restrict__ lev, int npt,
                                const int *__restrict__ nbox_of, Consts c) {
  for (int ib = blockIdx.x * blockDim.x + threadIdx.x; ib < npt; ib += gridDim.x * blockDim.x) {
    int i = S.nq0[ib];
    int mb = nbox_of[ib];
    double xi = S.x0[i], yi = S.y0[i];
    int k0 = S.kb1[mb], k1 = k0 + S.bcnt[mb];
    bool hit = false;
    for (int k = k0; k < k1 && !hit; k++) {
      int isb = S.bnode[k];
      int is = S.nq0[isb];
      if (is == ib || is == i) continue;
      hit = surg_test(xi, yi, S.x0[is], S.y0[is], S.dx0[is], S.dy0[is],
                      S.dx0[is] * S.dx0[is] + S.dy0[is] * S.dy0[is], c);
    }
    S.pending[ib] = hit ? 1 : 0;
  }
}

__device__ __forceinline__ void mark(SurgState &S, int x, int ib, int iend) {
  if (x > ib && x <= iend) S.pending[x] = 1;
}

// Mark every later node whose tests may read node j's changed data.
__device__ void mark_affected(SurgState &S, const LevelDesc &L, int j, int ib, const Consts &c) {
  int cand[2] = {j, S.prev0[j]};
  for (int q = 0; q < 2; q++) {
    int e = cand[q];
    mark(S, e, ib, L.iend);
    // boxes listing the segment whose list entry is e
    int i = S.nq0[e];
    int mbx1, mbx2, mby1, mby2;
    seg_boxes(S.x0[i], S.y0[i], S.dx0[i], S.dy0[i], L, c, mbx1, mbx2, mby1, mby2);
    for (int mbx = mbx1; mbx <= mbx2; mbx++) {
      int mmbx = mbx % L.nbx;
      for (int mby = mby1; mby <= mby2; mby++) {
        int gb = L.boxbase + L.nby * mmbx + mby % L.nby;
        int s = S.nb1[gb], n = S.nbcnt[gb];
        for (int k = 0; k < n; k++) mark(S, S.nbnode[s + k], ib, L.iend);
      }
    }
  }
}

// One warp per level replays contours.f90:528-613 at pending nodes.
__global__ void k_sg_replay(SurgState S, const LevelDesc *__restrict__ lev, int nlev, Consts c,
                            int *nsurg) {
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (warp >= nlev) return;
  const LevelDesc L = lev[warp];
  volatile unsigned char *pend = S.pending;
  volatile double *xq = S.xq, *yq = S.yq, *dx = S.dx, *dy = S.dy, *dsq = S.dsq;
  volatile int *nextq = S.nextq;
  const double f12 = 0.5;
  int count = 0;
  long long pos = L.ibeg;
  while (pos <= L.iend) {
    long long idx = pos + lane;
    bool f = idx <= L.iend && pend[idx];
    unsigned b = __ballot_sync(0xffffffffu, f);
    if (!b) {
      pos += 32;
      continue;
    }
    const int ib = (int)(pos + __ffs(b) - 1);
    __syncwarp();
    int i = nextq[ib];
    double xi = xq[i], yi = yq[i];
    int mb = node_box(xi, yi, L, c);
    int k = S.kb1[mb];
    const int kend = k + S.bcnt[mb];
    while (k < kend) {
      int kk = k + lane;
      bool pass = false;
      if (kk < kend) {
        int isb = S.bnode[kk];
        int is = nextq[isb];
        if (!(is == ib || is == i)) pass = surg_test(xi, yi, xq[is], yq[is], dx[is], dy[is], dsq[is], c);
      }
      unsigned pb = __ballot_sync(0xffffffffu, pass);
      if (!pb) {
        k += 32;
        continue;
      }
      kk = k + __ffs(pb) - 1;
      int inew = 0;
      if (lane == 0) {
        int isb = S.bnode[kk];
        int is = nextq[isb];
        double xx = xq[is] - xq[i];
        double delx = xx - c.ellx * f_dint(xx * c.hlxi);
        double yy = yq[is] - yq[i];
        double dely = yy - c.elly * f_dint(yy * c.hlyi);
        double aa = delx * dx[is] + dely * dy[is];
        double dxa, dya;
        if (dsq[is] + 2.0 * aa < 0.0) {
          dxa = f12 * (delx + dx[is]);
          dya = f12 * (dely + dy[is]);
          isb = is;
          is = nextq[is];
        } else {
          dxa = f12 * delx;
          dya = f12 * dely;
        }
        xx = xq[i] + dxa;
        xq[i] = wrapp(xx, c.ellx, c.hlxi, c.oms);
        yy = yq[i] + dya;
        yq[i] = wrapp(yy, c.elly, c.hlyi, c.oms);
        dx[i] = dx[i] - dxa;
        dy[i] = dy[i] - dya;
        dsq[i] = dx[i] * dx[i] + dy[i] * dy[i];
        nextq[isb] = i;
        dx[isb] = dx[isb] - dxa;
        dy[isb] = dy[isb] - dya;
        dsq[isb] = dx[isb] * dx[isb] + dy[isb] * dy[isb];
        xq[is] = xq[i];
        yq[is] = yq[i];
        dx[is] = dx[is] + dxa;
        dy[is] = dy[is] + dya;
        dsq[is] = dx[is] * dx[is] + dy[is] * dy[is];
        nextq[ib] = is;
        dx[ib] = dx[ib] + dxa;
        dy[ib] = dy[ib] + dya;
        dsq[ib] = dx[ib] * dx[ib] + dy[ib] * dy[ib];
        int touched[4] = {i, is, isb, ib};
        for (int q = 0; q < 4; q++) mark_affected(S, L, touched[q], ib, c);
        inew = is;
        count++;
      }
      __threadfence_block();
      __syncwarp();
      i = __shfl_sync(0xffffffffu, inew, 0);
      xi = xq[i];
      yi = yq[i];
      if (i == ib) break;
      k = kk + 1;
    }
    pos = ib + 1;
  }
  if (lane == 0 && count) atomicAdd(nsurg, count);
}

// ---------------------------------------------------------------------------
// Rebuild: cycles of nextq -> walk-ordered contours (contours.f90:621-663)
// ---------------------------------------------------------------------------
__global__ void k_rb_flags(const int *__restrict__ nextq, int npt, int *__restrict__ st,
                           int *__restrict__ brk) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npt; i += gridDim.x * blockDim.x) {
    brk[i] = nextq[i] != i + 1;
    st[i] = (i == 0) || (nextq[i - 1] != i);
  }
}

__global__ void k_rb_runs(const int *__restrict__ st, const int *__restrict__ brk,
                          const int *__restrict__ sx, int npt, int *__restrict__ rid,
                          int *__restrict__ rs, int *__restrict__ re) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npt; i += gridDim.x * blockDim.x) {
    int r = sx[i] + st[i] - 1;
    rid[i] = r;
    if (st[i]) rs[r] = i;
    if (brk[i]) re[r] = i;
  }
}

__global__ void k_rb_runinit(const int *__restrict__ nextq, const int *__restrict__ rid,
                             const int *__restrict__ rs, const int *__restrict__ re, int R,
                             int *__restrict__ nr, int *__restrict__ lab, int *__restrict__ nrj) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < R; r += gridDim.x * blockDim.x) {
    int t = rid[nextq[re[r]]];
    nr[r] = t;
    nrj[r] = t;
    lab[r] = rs[r];
  }
}

__global__ void k_rb_minjump(const int *__restrict__ lab, const int *__restrict__ nrj, int R,
                             int *__restrict__ lab2, int *__restrict__ nrj2) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < R; r += gridDim.x * blockDim.x) {
    int n = nrj[r];
    lab2[r] = min(lab[r], lab[n]);
    nrj2[r] = nrj[n];
  }
}

__global__ void k_rb_succ(const int *__restrict__ lab, const int *__restrict__ rid,
                          const int *__restrict__ nr, const int *__restrict__ rs,
                          const int *__restrict__ re, int R, int *__restrict__ hr,
                          int *__restrict__ succ, long long *__restrict__ val,
                          int *__restrict__ ishead) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < R; r += gridDim.x * blockDim.x) {
    int h = rid[lab[r]];
    hr[r] = h;
    succ[r] = nr[r] == h ? -1 : nr[r];  // the cycle's last run ends the list
    val[r] = re[r] - rs[r] + 1;
    ishead[r] = h == r;
  }
}

__global__ void k_rb_sumjump(const long long *__restrict__ val, const int *__restrict__ succ, int R,
                             long long *__restrict__ val2, int *__restrict__ succ2) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < R; r += gridDim.x * blockDim.x) {
    int s = succ[r];
    val2[r] = val[r] + (s >= 0 ? val[s] : 0);
    succ2[r] = s >= 0 ? succ[s] : -1;
  }
}

__global__ void k_rb_cycles(const int *__restrict__ ishead, const int *__restrict__ cidx,
                            const long long *__restrict__ val, const int *__restrict__ rs,
                            const int *__restrict__ lvl, const LevelDesc *__restrict__ lev, int R,
                            int *__restrict__ clen, int *__restrict__ clev) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < R; r += gridDim.x * blockDim.x) {
    if (!ishead[r]) continue;
    int c = cidx[r];
    clen[c] = (int)val[r];
    clev[c] = lev[lvl[rs[r]]].levt;
  }
}

__global__ void k_rb_gather(const double *__restrict__ xq, const double *__restrict__ yq, int npt,
                            const int *__restrict__ rid, const int *__restrict__ rs,
                            const int *__restrict__ hr, const int *__restrict__ cidx,
                            const long long *__restrict__ val, const int *__restrict__ cst,
                            const int *__restrict__ clen, double *__restrict__ xw,
                            double *__restrict__ yw) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npt; i += gridDim.x * blockDim.x) {
    int r = rid[i];
    int c = cidx[hr[r]];
    long long off = (long long)clen[c] - val[r];
    long long pos = cst[c] + off + (i - rs[r]);
    xw[pos] = xq[i];
    yw[pos] = yq[i];
  }
}

// Final contour arrays and canonical links (contours.f90:645-680).
__global__ void k_rb_contours(const int *__restrict__ ocs, const int *__restrict__ olen,
                              const int *__restrict__ olev, int nq, int *__restrict__ i1q,
                              int *__restrict__ i2q, int *__restrict__ npq,
                              int *__restrict__ indq) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nq; j += gridDim.x * blockDim.x) {
    i1q[j] = ocs[j];
    i2q[j] = ocs[j] + olen[j] - 1;
    npq[j] = olen[j];
    indq[j] = olev[j];
  }
}

__global__ void k_rb_links(const int *__restrict__ ocs, const int *__restrict__ olen, int nq,
                           int npt, int *__restrict__ nextq) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npt; i += gridDim.x * blockDim.x) {
    int j = contour_of(ocs, nq, i);
    nextq[i] = i + 1 < ocs[j] + olen[j] ? i + 1 : ocs[j];
  }
}

__global__ void k_set_counts(Scalars *s, const int *cnt) {
  s->nq = cnt[0];
  s->nptq = cnt[1];
}

static inline int gs(long long work) {
  long long g = (work + 255) / 256;
  if (g < 1) g = 1;
  if (g > 148 * 16) g = 148 * 16;
  return (int)g;
}

// Walk-ordered contours of the current link array + renode + write back.
// Used by surgery; lvl/lev give each node's level.
static int rebuild_and_renode(casl_handle *h, Arena &ar, const int *lvl, const LevelDesc *dlev) {
  cudaStream_t st = h->stream;
  int npt = h->nptq;
  int *stf = ar.get<int>(npt), *brk = ar.get<int>(npt), *sx = ar.get<int>(npt);
  int *rid = ar.get<int>(npt), *tmpi = ar.get<int>(scan_tmp_elems(npt) + 4);
  int *dtot = ar.get<int>(8);
  if (ar.failed) return CASL_ENOMEM;
  int g = gs(npt);
  CASL_K(k_rb_flags, g, 256, 0, st)(h->nextq, npt, stf, brk);
  exclusive_scan<int>(st, stf, sx, npt, tmpi, dtot);
  int R = 0;
  cudaMemcpyAsync(&R, dtot, sizeof(int), cudaMemcpyDeviceToHost, st);
  cudaError_t e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return set_cuda_error(h, e);
  int *rs = ar.get<int>(R), *re = ar.get<int>(R), *nr = ar.get<int>(R), *lab = ar.get<int>(R);
  int *lab2 = ar.get<int>(R), *nrj = ar.get<int>(R), *nrj2 = ar.get<int>(R), *hr = ar.get<int>(R);
  int *succ = ar.get<int>(R), *succ2 = ar.get<int>(R), *ishead = ar.get<int>(R);
  int *cidx = ar.get<int>(R);
  long long *val = ar.get<long long>(R), *val2 = ar.get<long long>(R);
  if (ar.failed) return CASL_ENOMEM;
  CASL_K(k_rb_runs, g, 256, 0, st)(stf, brk, sx, npt, rid, rs, re);
  int gr = gs(R);
  CASL_K(k_rb_runinit, gr, 256, 0, st)(h->nextq, rid, rs, re, R, nr, lab, nrj);
  int rounds = 1;
  while ((1 << rounds) < R) rounds++;
  rounds++;
  for (int it = 0; it < rounds; it++) {
    CASL_K(k_rb_minjump, gr, 256, 0, st)(lab, nrj, R, lab2, nrj2);
    std::swap(lab, lab2);
    std::swap(nrj, nrj2);
  }
  CASL_K(k_rb_succ, gr, 256, 0, st)(lab, rid, nr, rs, re, R, hr, succ, val, ishead);
  for (int it = 0; it < rounds; it++) {
    CASL_K(k_rb_sumjump, gr, 256, 0, st)(val, succ, R, val2, succ2);
    std::swap(val, val2);
    std::swap(succ, succ2);
  }
  exclusive_scan<int>(st, ishead, cidx, R, tmpi, dtot + 1);
  int C = 0;
  cudaMemcpyAsync(&C, dtot + 1, sizeof(int), cudaMemcpyDeviceToHost, st);
  e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return set_cuda_error(h, e);
  int *clen = ar.get<int>(C), *clev = ar.get<int>(C), *cst = ar.get<int>(C);
  double *xw = ar.get<double>(npt), *yw = ar.get<double>(npt);
  if (ar.failed) return CASL_ENOMEM;
  CASL_K(k_rb_cycles, gr, 256, 0, st)(ishead, cidx, val, rs, lvl, dlev, R, clen, clev);
  exclusive_scan<int>(st, clen, cst, C, tmpi, dtot + 2);
  CASL_K(k_rb_gather, g, 256, 0, st)(h->xq, h->yq, npt, rid, rs, hr, cidx, val, cst, clen, xw, yw);
  int rc = check_launch(h);
  if (rc) return rc;
  // renode every cycle; write straight into the node arrays
  RenodeIn in{xw, yw, cst, clen, clev, C, npt};
  RenodeOut out{};
  out.xo = h->xqi;  // node-sized scratch of the RK step, free between steps
  out.yo = h->yqi;
  out.ocs = ar.get<int>(C); out.olen = ar.get<int>(C); out.olev = ar.get<int>(C);
  out.cap = h->npm;
  out.d_counts = ar.get<int>(4);
  if (ar.failed) return CASL_ENOMEM;
  rc = renode_batch(h, ar, in, out, RENODE_SURGERY);
  if (rc) return rc;
  int hc[3];
  cudaMemcpyAsync(hc, out.d_counts, 3 * sizeof(int), cudaMemcpyDeviceToHost, st);
  e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return set_cuda_error(h, e);
  int nq = hc[0], nptn = hc[1];
  if (nq > h->nm || nptn > h->npm) return CASL_ECAPACITY;
  if (nptn > 0) {
    cudaMemcpyAsync(h->xq, out.xo, (size_t)nptn * sizeof(double), cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(h->yq, out.yo, (size_t)nptn * sizeof(double), cudaMemcpyDeviceToDevice, st);
  }
  if (nq > 0) {
    CASL_K(k_rb_contours, gs(nq), 256, 0, st)(out.ocs, out.olen, out.olev, nq, h->i1q, h->i2q, h->npq,
                                          h->indq);
    CASL_K(k_rb_links, gs(nptn), 256, 0, st)(out.ocs, out.olen, nq, nptn, h->nextq);
  }
  CASL_K(k_set_counts, 1, 1, 0, st)(h->scal, out.d_counts);
  rc = check_launch(h);
  if (rc) return rc;
  h->nq = nq;
  h->nptq = nptn;
  h->contex = nptn > 0;
  return CASL_OK;
}

int surgery_dev(casl_handle *h) {
  if (h->nq == 0 || h->nptq == 0) return CASL_OK;
  cudaStream_t st = h->stream;
  const Consts &c = h->c;
  int nq = h->nq, npt = h->nptq;
  // Levels (contours.f90:374-394) and box dimensions (contours.f90:429-454),
  // on the host from the contour table.
  std::vector<int> indq(nq), i1q(nq), i2q(nq);
  cudaMemcpyAsync(indq.data(), h->indq, nq * sizeof(int), cudaMemcpyDeviceToHost, st);
  cudaMemcpyAsync(i1q.data(), h->i1q, nq * sizeof(int), cudaMemcpyDeviceToHost, st);
  cudaMemcpyAsync(i2q.data(), h->i2q, nq * sizeof(int), cudaMemcpyDeviceToHost, st);
  cudaError_t e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return set_cuda_error(h, e);
  std::vector<LevelDesc> lev;
  {
    int levp = indq[0], jq1 = 0;
    auto push = [&](int j1, int j2, int levt) {
      LevelDesc L{};
      L.ibeg = i1q[j1];
      L.iend = i2q[j2];
      L.levt = levt;
      lev.push_back(L);
    };
    for (int j = 1; j < nq; j++) {
      if (indq[j] > levp) {
        push(jq1, j - 1, levp);
        jq1 = j;
        levp = indq[j];
      }
    }
    push(jq1, nq - 1, levp);
  }
  long long nbox = 0;
  for (auto &L : lev) {
    if (L.ibeg < 0 || L.iend >= npt || L.iend < L.ibeg) return CASL_EINVAL;
    int nptlev = L.iend - L.ibeg + 1;
    double fnq = (double)nptlev;
    double fnbx = 1.2 * sqrt(fnq * c.aspect);
    double fnby = fnbx / c.aspect;
    int nbx = (int)llround(fnbx);
    nbx = std::max(std::min(nbx, c.nx), 1);
    int nby = (int)llround(fnby);
    nby = std::max(std::min(nby, c.ny), 1);
    L.nbx = nbx;
    L.nby = nby;
    L.bwxi = c.oms * (double)nbx / c.ellx;
    L.bwyi = c.oms * (double)nby / c.elly;
    L.boxbase = (int)nbox;
    nbox += (long long)nbx * nby;
  }
  int nlev = (int)lev.size();
  // scratch
  size_t need = (size_t)npt * 560 + (size_t)nbox * 40 + (size_t)nq * 256 + ((size_t)64 << 20);
  int rc = ensure_scratch(h, need);
  if (rc) return rc;
  Arena ar{(char *)h->sx, h->sx_bytes, 0};
  LevelDesc *dlev = ar.get<LevelDesc>(nlev);
  int *endnext = ar.get<int>(npt), *lvl = ar.get<int>(npt);
  double *dx = ar.get<double>(npt), *dy = ar.get<double>(npt), *dsq = ar.get<double>(npt);
  double *x0 = ar.get<double>(npt), *y0 = ar.get<double>(npt);
  double *dx0 = ar.get<double>(npt), *dy0 = ar.get<double>(npt);
  int *nq0 = ar.get<int>(npt), *prev0 = ar.get<int>(npt);
  unsigned char *pending = ar.get<unsigned char>(npt);
  int *ecount = ar.get<int>(npt), *eoff = ar.get<int>(npt), *nbox_of = ar.get<int>(npt);
  int *bcnt = ar.get<int>(nbox), *kb1 = ar.get<int>(nbox), *cursor = ar.get<int>(nbox);
  int *nbcnt = ar.get<int>(nbox), *nb1 = ar.get<int>(nbox), *nbnode = ar.get<int>(npt);
  int *tmpi = ar.get<int>(scan_tmp_elems(std::max<long long>(npt, nbox)) + 4);
  int *dtot = ar.get<int>(8);
  if (ar.failed) return CASL_ENOMEM;
  cudaMemcpyAsync(dlev, lev.data(), nlev * sizeof(LevelDesc), cudaMemcpyHostToDevice, st);
  cudaMemsetAsync(endnext, 0xff, (size_t)npt * sizeof(int), st);
  cudaMemsetAsync(bcnt, 0, (size_t)nbox * sizeof(int), st);
  cudaMemsetAsync(nbcnt, 0, (size_t)nbox * sizeof(int), st);
  cudaMemsetAsync(&h->scal->error, 0, sizeof(int), st);
  int g = gs(npt);
  CASL_K(k_sg_endnext, gs(nq), 256, 0, st)(h->i1q, h->i2q, nq, endnext);
  CASL_K(k_sg_level_of, g, 256, 0, st)(dlev, nlev, npt, lvl);
  CASL_K(k_sg_init, g, 256, 0, st)(h->xq, h->yq, h->nextq, endnext, npt, dx, dy, dsq, x0, y0, dx0, dy0,
                               nq0, prev0, pending, c, &h->scal->error);
  SurgState S{};
  S.xq = h->xq; S.yq = h->yq; S.dx = dx; S.dy = dy; S.dsq = dsq; S.nextq = h->nextq;
  S.x0 = x0; S.y0 = y0; S.dx0 = dx0; S.dy0 = dy0; S.nq0 = nq0; S.prev0 = prev0; S.lvl = lvl;
  S.pending = pending;
  CASL_K(k_sg_count_entries, g, 256, 0, st)(S, dlev, npt, ecount, nbox_of, nbcnt, c);
  exclusive_scan<int>(st, ecount, eoff, npt, tmpi, dtot);
  int ne = 0;
  cudaMemcpyAsync(&ne, dtot, sizeof(int), cudaMemcpyDeviceToHost, st);
  int herr = 0;
  cudaMemcpyAsync(&herr, &h->scal->error, sizeof(int), cudaMemcpyDeviceToHost, st);
  e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return set_cuda_error(h, e);
  if (herr) return herr;
  int *ebox = ar.get<int>(ne), *eib = ar.get<int>(ne), *bnode = ar.get<int>(ne);
  if (ar.failed) return CASL_ENOMEM;
  CASL_K(k_sg_emit, g, 256, 0, st)(S, dlev, npt, eoff, ebox, eib, bcnt, c);
  exclusive_scan<int>(st, bcnt, kb1, nbox, tmpi, dtot + 1);
  cudaMemsetAsync(cursor, 0, (size_t)nbox * sizeof(int), st);
  CASL_K(k_sg_place, gs(ne), 256, 0, st)(ebox, eib, ne, kb1, cursor, bnode);
  CASL_K(k_sg_sort_boxes, gs(nbox), 256, 0, st)(kb1, bcnt, (int)nbox, bnode);
  exclusive_scan<int>(st, nbcnt, nb1, nbox, tmpi, dtot + 2);
  cudaMemsetAsync(cursor, 0, (size_t)nbox * sizeof(int), st);
  CASL_K(k_sg_place_nodes, g, 256, 0, st)(nbox_of, npt, nb1, cursor, nbnode);
  S.kb1 = kb1; S.bcnt = bcnt; S.bnode = bnode; S.nb1 = nb1; S.nbcnt = nbcnt; S.nbnode = nbnode;
  CASL_K(k_sg_candidates, g, 256, 0, st)(S, dlev, npt, nbox_of, c);
  int *nsurg = dtot + 4;
  cudaMemsetAsync(nsurg, 0, sizeof(int), st);
  CASL_K(k_sg_replay, (nlev * 32 + 127) / 128, 128, 0, st)(S, dlev, nlev, c, nsurg);
  rc = check_launch(h);
  if (rc) return rc;
  return rebuild_and_renode(h, ar, lvl, dlev);
}

// Renode of one contour supplied by the host (casl_renode).
int renode_host(casl_handle *h, const double *xd, const double *yd, int npd, double *xr,
                double *yr, int cap, int *npr) {
  cudaStream_t st = h->stream;
  size_t need = (size_t)npd * 200 + (size_t)cap * 16 + ((size_t)16 << 20);
  int rc = ensure_scratch(h, need);
  if (rc) return rc;
  Arena ar{(char *)h->sx, h->sx_bytes, 0};
  double *xw = ar.get<double>(npd), *yw = ar.get<double>(npd);
  double *xo = ar.get<double>(cap + 1), *yo = ar.get<double>(cap + 1);
  int *cs = ar.get<int>(1), *len = ar.get<int>(1);
  RenodeOut out{};
  out.xo = xo; out.yo = yo;
  out.ocs = ar.get<int>(1); out.olen = ar.get<int>(1); out.olev = ar.get<int>(1);
  out.cap = cap;
  out.d_counts = ar.get<int>(4);
  if (ar.failed) return CASL_ENOMEM;
  int z = 0;
  CASL_CUDA_TRY(cudaMemcpyAsync(xw, xd, npd * sizeof(double), cudaMemcpyHostToDevice, st));
  CASL_CUDA_TRY(cudaMemcpyAsync(yw, yd, npd * sizeof(double), cudaMemcpyHostToDevice, st));
  CASL_CUDA_TRY(cudaMemcpyAsync(cs, &z, sizeof(int), cudaMemcpyHostToDevice, st));
  CASL_CUDA_TRY(cudaMemcpyAsync(len, &npd, sizeof(int), cudaMemcpyHostToDevice, st));
  RenodeIn in{xw, yw, cs, len, nullptr, 1, npd};
  rc = renode_batch(h, ar, in, out, RENODE_PLAIN);
  if (rc) return rc;
  int hc[3];
  CASL_CUDA_TRY(cudaMemcpyAsync(hc, out.d_counts, 3 * sizeof(int), cudaMemcpyDeviceToHost, st));
  CASL_CUDA_TRY(cudaStreamSynchronize(st));
  *npr = hc[1];
  if (hc[1] > 0) {
    CASL_CUDA_TRY(cudaMemcpyAsync(xr, xo, hc[1] * sizeof(double), cudaMemcpyDeviceToHost, st));
    CASL_CUDA_TRY(cudaMemcpyAsync(yr, yo, hc[1] * sizeof(double), cudaMemcpyDeviceToHost, st));
    CASL_CUDA_TRY(cudaStreamSynchronize(st));
  }
  return check_launch(h);
}

}  // namespace casl
