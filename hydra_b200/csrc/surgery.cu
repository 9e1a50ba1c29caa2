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
#include <limits.h>
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
  const int *bnq;                      // nq0 of each bnode entry
  const int *nb1, *nbcnt, *nbnode;     // nodes located per box
  unsigned char *pending;
  // one bit per window of 512 nodes (a word per 16384) set wherever a
  // pending flag is set, so the replay skips empty windows a word at a time
  unsigned int *wsum;
};

__device__ __forceinline__ void set_pending(const SurgState &S, int x) {
  S.pending[x] = 1;
  atomicOr(&S.wsum[x >> 14], 1u << ((x >> 9) & 31));
}

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


// --- levels (contours.f90:374-394) and box counts (contours.f90:429-454) ----
// A new level starts where indq increases; contours arrive sorted by level.




// The level table in one block (levels are few, contours ~1e4): level
// starts where indq increases, their ranks, each level's node range, box
// counts nint(1.2 sqrt(N_lev)) per side (contours.f90:403-416) and the
// levels' first global boxes; and endnext, each contour's last node linked
// to its first (the rest of endnext is -1 on entry).  dtot[0] = levels,
// dtot[1] = boxes.
__global__ void __launch_bounds__(SCAN_BLOCK) k_lv_all(const int *__restrict__ i1q,
                                                       const int *__restrict__ i2q,
                                                       const int *__restrict__ indq, int nq,
                                                       int npt, Consts c,
                                                       LevelDesc *__restrict__ lev,
                                                       int *__restrict__ lidx,
                                                       int *__restrict__ endnext,
                                                       int *__restrict__ dtot,
                                                       long long nbox_cap,
                                                       int *__restrict__ err) {
  CASL_PDL_ENTRY();
  __shared__ int tot, carry;
  const int tid = threadIdx.x;
  // each thread takes a run of consecutive contours: it counts the level
  // starts in its run, one block scan numbers them, and a second pass over
  // the run writes the levels (two rounds of loads instead of one per
  // 1024 contours)
  const int per = (nq + SCAN_BLOCK - 1) / SCAN_BLOCK;
  const int j0 = min(nq, tid * per), j1 = min(nq, j0 + per);
  int cnt = 0;
  {
    int prev = j0 > 0 ? indq[j0 - 1] : 0;
    for (int j = j0; j < j1; j++) {
      const int v = indq[j];
      cnt += j == 0 || v > prev;
      if (j > 0 && v < prev) atomicExch(err, CASL_EINVAL);
      prev = v;
    }
  }
  int lv = block_excl_scan<int>(cnt, &tot) - 1;
  const int nlev = tot;
  {
    int prev = j0 > 0 ? indq[j0 - 1] : 0;
    for (int j = j0; j < j1; j++) {
      const int v = indq[j], a = i1q[j], b = i2q[j];
      const bool first = j == 0 || v > prev;
      lv += first;
      lidx[j] = lv;  // the level of contour j
      endnext[b] = a;  // a contour's last node links back to its first
      if (first) {
        lev[lv].ibeg = a;
        lev[lv].levt = v;
      }
      if (j == nq - 1 || indq[j + 1] > v) lev[lv].iend = b;
      prev = v;
    }
  }
  __syncthreads();
  if (tid == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < nlev; base += SCAN_BLOCK) {
    const int L = base + tid;
    int nb = 0;
    LevelDesc d{};
    bool ok = false;
    if (L < nlev) {
      d = lev[L];
      if (d.ibeg < 0 || d.iend >= npt || d.iend < d.ibeg) {
        atomicExch(err, CASL_EINVAL);
      } else {
        ok = true;
        double fnq = (double)(d.iend - d.ibeg + 1);
        double fnbx = 1.2 * sqrt(fnq * c.aspect);
        double fnby = fnbx / c.aspect;
        int nbx = (int)llround(fnbx);
        nbx = max(min(nbx, c.nx), 1);
        int nby = (int)llround(fnby);
        nby = max(min(nby, c.ny), 1);
        d.nbx = nbx;
        d.nby = nby;
        d.bwxi = c.oms * (double)nbx / c.ellx;
        d.bwyi = c.oms * (double)nby / c.elly;
        nb = nbx * nby;
      }
    }
    const int ex = block_excl_scan<int>(nb, &tot) + carry;
    if (ok) {
      d.boxbase = ex;
      lev[L] = d;
    }
    __syncthreads();
    if (tid == 0) carry += tot;
    __syncthreads();
  }
  if (tid == 0) {
    dtot[0] = nlev;
    dtot[1] = carry;
    if ((long long)carry > nbox_cap) atomicExch(err, CASL_ECAPACITY);
  }
}



// work arrays dx, dy, dsq (contours.f90:397-415) and the original copies
__global__ void k_sg_init(const double *__restrict__ xq, const double *__restrict__ yq,
                          const int *__restrict__ nextq, const int *__restrict__ endnext, int npt,
                          double *dx, double *dy, double *dsq, double *x0, double *y0,
                          double *dx0, double *dy0, int *nq0, int *prev0, unsigned char *pending,
                          const LevelDesc *__restrict__ lev, const int *__restrict__ nlev_dev,
                          int *__restrict__ lvl, Consts c, int *err) {
  CASL_PDL_ENTRY();
  const int nlev = *nlev_dev;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npt; i += gridDim.x * blockDim.x) {
    {
      // the node's level: the last level starting at or below i
      int lo = 0, hi = nlev - 1;
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (lev[mid].ibeg <= i) lo = mid; else hi = mid - 1;
      }
      lvl[i] = lo;
    }
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

// Per segment: the number of box entries it makes, and where they start
// relative to its block's share of the entries.  Block b takes the nodes
// [b*chunk, (b+1)*chunk) in steps of blockDim.x with a running carry, then
// takes its share of the entry array with one atomic on the running total
// (bbase[b]); the entries' order in memory is free, since every box list is
// read as a set.
__global__ void k_sg_count_entries(SurgState S, const LevelDesc *__restrict__ lev, int npt,
                                   int chunk, int *__restrict__ ecount, int *__restrict__ eoff,
                                   int *__restrict__ bbase, int *__restrict__ ne_tot,
                                   int *__restrict__ nbox_of, int *__restrict__ nbcnt, Consts c) {
  CASL_PDL_ENTRY();
  __shared__ int btot;
  const int b0 = blockIdx.x * chunk, b1 = min(npt, b0 + chunk);
  int carry = 0;
  for (int base = b0; base < b1; base += blockDim.x) {
    const int ib = base + threadIdx.x;
    int cnt = 0;
    if (ib < b1) {
      LevelDesc L = lev[S.lvl[ib]];
      int i = S.nq0[ib];
      int mbx1, mbx2, mby1, mby2;
      seg_boxes(S.x0[i], S.y0[i], S.dx0[i], S.dy0[i], L, c, mbx1, mbx2, mby1, mby2);
      cnt = (mbx2 - mbx1 + 1) * (mby2 - mby1 + 1);
      ecount[ib] = cnt;
      int nb = node_box(S.x0[i], S.y0[i], L, c);
      nbox_of[ib] = nb;
      red_add_s32(&nbcnt[nb], 1);
    }
    const int ex = block_excl_scan_any<int>(cnt, &btot);
    if (ib < b1) eoff[ib] = carry + ex;
    carry += btot;
  }
  if (threadIdx.x == 0) bbase[blockIdx.x] = atomicAdd(ne_tot, carry);
}

// Start of every box's segment list and of its node list.  Block b takes
// the boxes [b*chunk, (b+1)*chunk): it sums their counts, takes its share
// of both lists with one atomic each (box order in memory is free), then
// scans the counts again (from L2) and writes each start twice, the start
// itself and the placement cursor.
__global__ void __launch_bounds__(1024) k_sg_box_alloc(const int *__restrict__ bcnt,
                                                       const int *__restrict__ nbcnt,
                                                       const int *__restrict__ nbox_dev,
                                                       long long nbox_cap, long long chunk,
                                                       int *__restrict__ kb1,
                                                       int *__restrict__ cb,
                                                       int *__restrict__ nb1,
                                                       int *__restrict__ cn,
                                                       int *__restrict__ tot) {
  CASL_PDL_ENTRY();
  __shared__ unsigned long long btot;
  __shared__ int bb[2];
  const long long nbox = *nbox_dev < nbox_cap ? (long long)*nbox_dev : nbox_cap;
  const long long g0 = (long long)blockIdx.x * chunk;
  const long long g1 = g0 + chunk < nbox ? g0 + chunk : nbox;
  if (g0 >= g1) return;
  // both counts in one word: segment entries in the high half, nodes in the
  // low half (each total stays below 2^31)
  auto pack = [&](long long gb) -> unsigned long long {
    return gb < g1 ? ((unsigned long long)bcnt[gb] << 32) | (unsigned)nbcnt[gb] : 0ull;
  };
  unsigned long long sum = 0;
  for (long long gb = g0 + threadIdx.x; gb < g1; gb += blockDim.x) sum += pack(gb);
  block_excl_scan_any<unsigned long long>(sum, &btot);
  if (threadIdx.x == 0) {
    bb[0] = atomicAdd(&tot[0], (int)(btot >> 32));
    bb[1] = atomicAdd(&tot[1], (int)(btot & 0xffffffffu));
  }
  __syncthreads();
  unsigned long long carry = ((unsigned long long)(unsigned)bb[0] << 32) | (unsigned)bb[1];
  for (long long base = g0; base < g1; base += blockDim.x) {
    const long long gb = base + threadIdx.x;
    const unsigned long long ex = block_excl_scan_any<unsigned long long>(pack(gb), &btot) + carry;
    if (gb < g1) {
      const int k = (int)(ex >> 32), m = (int)(ex & 0xffffffffu);
      kb1[gb] = k;
      cb[gb] = k;
      nb1[gb] = m;
      cn[gb] = m;
    }
    carry += btot;
  }
}

__global__ void k_sg_emit(SurgState S, const LevelDesc *__restrict__ lev, int npt,
                          const int *__restrict__ eoff, const int *__restrict__ bbase, int chunk,
                          const int *__restrict__ ecount,
                          long long ne_cap, int *__restrict__ ebox, int *__restrict__ eib,
                          int *__restrict__ bcnt, Consts c, int *__restrict__ err) {
  CASL_PDL_ENTRY();
  for (int ib = blockIdx.x * blockDim.x + threadIdx.x; ib < npt; ib += gridDim.x * blockDim.x) {
    LevelDesc L = lev[S.lvl[ib]];
    int i = S.nq0[ib];
    int mbx1, mbx2, mby1, mby2;
    seg_boxes(S.x0[i], S.y0[i], S.dx0[i], S.dy0[i], L, c, mbx1, mbx2, mby1, mby2);
    long long e = (long long)eoff[ib] + bbase[ib / chunk];
    // Past the capacity nothing is written (CASL_ECAPACITY is raised): the
    // offsets tile [0, total) densely, so every entry below the capacity is
    // written, and the box counts count exactly the entries written.
    if (e + ecount[ib] > ne_cap) atomicExch(err, CASL_ECAPACITY);
    for (int mbx = mbx1; mbx <= mbx2; mbx++) {
      int mmbx = mbx % L.nbx;
      for (int mby = mby1; mby <= mby2; mby++) {
        int gb = L.boxbase + L.nby * mmbx + mby % L.nby;
        if (e < ne_cap) {
          ebox[e] = gb;
          eib[e] = ib;
          red_add_s32(&bcnt[gb], 1);
        }
        e++;
      }
    }
  }
}

__global__ void k_sg_place(const int *__restrict__ ebox, const int *__restrict__ eib,
                           const int *__restrict__ ne_dev, long long ne_cap,
                           int *__restrict__ cursor, const int *__restrict__ nq0,
                           int *__restrict__ bnode, int *__restrict__ bnq) {
  CASL_PDL_ENTRY();
  // the emit pass wrote the entries below the capacity only
  const long long ne = *ne_dev < ne_cap ? (long long)*ne_dev : ne_cap;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < ne;
       e += (long long)gridDim.x * blockDim.x) {
    int gb = ebox[e];
    int pos = atomicAdd(&cursor[gb], 1);  // starts at the box's list start
    const int isb = eib[e];
    bnode[pos] = isb;
    bnq[pos] = nq0[isb];  // the candidate search reads the segment's end node directly
  }
}

__global__ void k_sg_place_nodes(const int *__restrict__ nbox_of, int npt,
                                 int *__restrict__ cursor,
                                 int *__restrict__ nbnode) {
  CASL_PDL_ENTRY();
  for (int ib = blockIdx.x * blockDim.x + threadIdx.x; ib < npt; ib += gridDim.x * blockDim.x) {
    int gb = nbox_of[ib];
    nbnode[atomicAdd(&cursor[gb], 1)] = ib;  // cursor starts at the box's list start
  }
}

// Restore the reference's per-box order (ascending node before the segment).
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
  CASL_PDL_ENTRY();
  for (int ib = blockIdx.x * blockDim.x + threadIdx.x; ib < npt; ib += gridDim.x * blockDim.x) {
    int i = S.nq0[ib];
    int mb = nbox_of[ib];
    double xi = S.x0[i], yi = S.y0[i];
    int k0 = S.kb1[mb], k1 = k0 + S.bcnt[mb];
    bool hit = false;
    // the next entry's node index is loaded while this one is tested
    int isn = k0 < k1 ? S.bnq[k0] : 0;
    for (int k = k0; k < k1 && !hit; k++) {
      const int is = isn;
      if (k + 1 < k1) isn = S.bnq[k + 1];
      if (is == ib || is == i) continue;
      const double dxs = S.dx0[is], dys = S.dy0[is];
      hit = surg_test(xi, yi, S.x0[is], S.y0[is], dxs, dys, dxs * dxs + dys * dys, c);
    }
    S.pending[ib] = hit ? 1 : 0;
    if (hit) atomicOr(&S.wsum[ib >> 14], 1u << ((ib >> 9) & 31));
  }
}

__device__ __forceinline__ void mark(SurgState &S, int x, int ib, int iend) {
  if (x > ib && x <= iend) set_pending(S, x);
}

// Mark every later node whose tests may read node j's changed data.  Called
// by all 32 lanes of the level's warp with the same j: the loops over boxes
// are uniform and the entries of each box are split across the lanes.
__device__ void mark_affected(SurgState &S, const LevelDesc &L, int j, int ib, const Consts &c,
                              int lane) {
  int cand[2] = {j, S.prev0[j]};
  for (int q = 0; q < 2; q++) {
    int e = cand[q];
    if (lane == 0) mark(S, e, ib, L.iend);
    // boxes listing the segment whose list entry is e
    int i = S.nq0[e];
    int mbx1, mbx2, mby1, mby2;
    seg_boxes(S.x0[i], S.y0[i], S.dx0[i], S.dy0[i], L, c, mbx1, mbx2, mby1, mby2);
    for (int mbx = mbx1; mbx <= mbx2; mbx++) {
      int mmbx = mbx % L.nbx;
      for (int mby = mby1; mby <= mby2; mby++) {
        int gb = L.boxbase + L.nby * mmbx + mby % L.nby;
        int s = S.nb1[gb], n = S.nbcnt[gb];
        for (int k = lane; k < n; k += 32) mark(S, S.nbnode[s + k], ib, L.iend);
      }
    }
  }
}

// One warp per level replays contours.f90:528-613 at pending nodes.
__global__ void k_sg_replay(SurgState S, const LevelDesc *__restrict__ lev,
                            const int *__restrict__ nlev_dev, Consts c, int *nsurg,
                            int *__restrict__ stats) {
  CASL_PDL_ENTRY();
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (warp >= *nlev_dev) return;
  const LevelDesc L = lev[warp];
  // Every node, flag and box entry this warp reads or writes belongs to its
  // own level, so no other warp touches them: lane 0's updates reach the
  // other lanes through this SM's L1 after __syncwarp(), and plain cached
  // loads are coherent here.
  const unsigned char *pend = S.pending;
  double *xq = S.xq, *yq = S.yq, *dx = S.dx, *dy = S.dy, *dsq = S.dsq;
  int *nextq = S.nextq;
  const double f12 = 0.5;
  int count = 0, npend = 0;
  long long pos = L.ibeg;
  while (pos <= L.iend) {
    int ib;
    {
      // skip the 512-node windows whose summary bit is clear (read from L2:
      // this warp's own marks arrive there by atomics)
      const long long W = pos >> 9;
      const unsigned sw = __ldcg(&S.wsum[W >> 5]) >> (W & 31);
      if (!sw) {
        pos = ((W >> 5) + 1) << 14;
        continue;
      }
      const int d = __ffs(sw) - 1;
      if (d > 0) {
        pos = (W + d) << 9;
        if (pos > L.iend) break;
      }
    }
    // Windows start at the 16-aligned position at or below pos, so the wide
    // path is taken whatever the level's first node; flags below pos (already
    // visited, or another level's) are masked out.
    const long long base = pos & ~15LL;
    if (base + 512 <= (long long)L.iend + 1) {
      // 512 flags per step: one 16-byte load per lane
      uint4 v = reinterpret_cast<const uint4 *>(pend + base)[lane];
      if (lane == 0 && pos > base) {
        const int sh = (int)(pos - base);  // 1..15 leading bytes to drop
        unsigned w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int q = 0; q < 4; q++) {
          const int drop = sh - 4 * q;  // bytes of word q below pos
          if (drop >= 4) w[q] = 0u;
          else if (drop > 0) w[q] &= ~0u << (8 * drop);
        }
        v = make_uint4(w[0], w[1], w[2], w[3]);
      }
      unsigned b = __ballot_sync(0xffffffffu, (v.x | v.y | v.z | v.w) != 0u);
      if (!b) {
        pos = base + 512;
        continue;
      }
      const int f = __ffs(b) - 1;
      int off = 0;
      if (lane == f) {
        unsigned w[4] = {v.x, v.y, v.z, v.w};
        for (int q = 0; q < 4; q++)
          if (w[q]) {
            off = 4 * q + (__ffs(w[q]) - 1) / 8;
            break;
          }
      }
      off = __shfl_sync(0xffffffffu, off, f);
      ib = (int)(base + 16 * f + off);
    } else {
      long long idx = base + lane;
      bool fl = idx >= pos && idx <= L.iend && pend[idx];
      unsigned b = __ballot_sync(0xffffffffu, fl);
      if (!b) {
        pos = base + 32;
        continue;
      }
      ib = (int)(base + __ffs(b) - 1);
    }
    __syncwarp();
    npend++;
    int i = nextq[ib];
    double xi = xq[i], yi = yq[i];
    int mb = node_box(xi, yi, L, c);
    const int kbeg = S.kb1[mb];
    const int kend = kbeg + S.bcnt[mb];
    // The reference walks the box's segments in list order and continues
    // after each reconnection with the moved node.  The box list is stored
    // unordered, so each round takes the passing segment with the smallest
    // list index above the last one taken.
    int thr = -1;
    while (true) {
      int best = INT_MAX;
      for (int kk = kbeg + lane; kk < kend; kk += 32) {
        int isb = S.bnode[kk];
        if (isb > thr && isb < best) {
          int is = nextq[isb];
          if (!(is == ib || is == i) && surg_test(xi, yi, xq[is], yq[is], dx[is], dy[is], dsq[is], c))
            best = isb;
        }
      }
      for (int o = 16; o > 0; o >>= 1) best = min(best, __shfl_xor_sync(0xffffffffu, best, o));
      if (best == INT_MAX) break;
      int inew = 0, tsb = 0;
      if (lane == 0) {
        int isb = best;
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
        tsb = isb;
        inew = is;
        count++;
      }
      __syncwarp();  // lane 0's moves are visible to the whole warp
      const int is_new = __shfl_sync(0xffffffffu, inew, 0);
      const int isb_new = __shfl_sync(0xffffffffu, tsb, 0);
      {
        const int touched[4] = {i, is_new, isb_new, ib};
        for (int q = 0; q < 4; q++) mark_affected(S, L, touched[q], ib, c, lane);
      }
      __syncwarp();  // marks visible before the next flag scan
      i = is_new;
      xi = xq[i];
      yi = yq[i];
      if (i == ib) break;
      thr = best;
    }
    pos = ib + 1;
  }
  if (lane == 0 && count) atomicAdd(nsurg, count);
  if (stats && lane == 0) {  // trace only: pending nodes visited, surgeries
    stats[2 * warp] = npend;
    stats[2 * warp + 1] = count;
  }
}

// ---------------------------------------------------------------------------
// Rebuild: cycles of nextq -> walk-ordered contours (contours.f90:621-663)
// ---------------------------------------------------------------------------
__global__ void k_rb_flags(const int *__restrict__ nextq, int npt, int *__restrict__ st,
                           int *__restrict__ brk) {
  CASL_PDL_ENTRY();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npt; i += gridDim.x * blockDim.x) {
    brk[i] = nextq[i] != i + 1;
    st[i] = (i == 0) || (nextq[i - 1] != i);
  }
}

__global__ void k_rb_runs(const int *__restrict__ st, const int *__restrict__ brk,
                          const int *__restrict__ sx, int npt, int *__restrict__ rid,
                          int *__restrict__ rs, int *__restrict__ re) {
  CASL_PDL_ENTRY();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npt; i += gridDim.x * blockDim.x) {
    int r = sx[i] + st[i] - 1;
    rid[i] = r;
    if (st[i]) rs[r] = i;
    if (brk[i]) re[r] = i;
  }
}











// All run-level cycle work in one block.  A contour no reconnection touched
// is a single run that points to itself and is finished at once; pointer
// jumping (min label, then list ranking) runs over the few remaining runs
// only, rounds separated by block barriers.
// Every run: its successor run; a run that closes on itself is a whole
// contour (head, length); the others (the few runs surgery cut and joined)
// go to the multi list for k_rb_cycles_block.  Grid-wide.
__global__ void k_rb_cycles_pre(const int *__restrict__ nextq, const int *__restrict__ rid,
                                const int *__restrict__ rs, const int *__restrict__ re,
                                const int *__restrict__ R_dev, int *__restrict__ nr,
                                int *__restrict__ lab, int *__restrict__ nrj,
                                int *__restrict__ hr, long long *__restrict__ val,
                                long long *__restrict__ val2, int *__restrict__ ishead,
                                int *__restrict__ multi, int *__restrict__ nmulti) {
  CASL_PDL_ENTRY();
  const int R = *R_dev;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < R; r += gridDim.x * blockDim.x) {
    const int t = rid[nextq[re[r]]];
    nr[r] = t;
    const long long len = re[r] - rs[r] + 1;
    lab[r] = rs[r];
    if (t == r) {  // a whole contour
      hr[r] = r;
      ishead[r] = 1;
      val[r] = len;
      val2[r] = len;
    } else {
      nrj[r] = t;
      multi[atomicAdd(nmulti, 1)] = r;
    }
  }
}

// The cycles through the multi-run list: one block, pointer jumping over
// the M runs in shared order.
__global__ void __launch_bounds__(1024) k_rb_cycles_block(
    const int *__restrict__ nextq, const int *__restrict__ rid, const int *__restrict__ rs,
    const int *__restrict__ re, const int *__restrict__ R_dev, int *__restrict__ nr,
    int *lab, int *lab2, int *nrj, int *nrj2, int *__restrict__ hr, int *succ, int *succ2,
    long long *val, long long *val2, int *__restrict__ ishead, int *__restrict__ multi,
    long long **valout, const int *__restrict__ nmulti) {
  CASL_PDL_ENTRY();
  const int M = *nmulti;
  int rounds = 1;
  while ((1 << rounds) < M) rounds++;
  rounds++;
  for (int it = 0; it < rounds && M > 0; it++) {
    for (int q = threadIdx.x; q < M; q += blockDim.x) {
      int r = multi[q];
      int n = nrj[r];
      lab2[r] = min(lab[r], lab[n]);
      nrj2[r] = nrj[n];
    }
    __syncthreads();
    for (int q = threadIdx.x; q < M; q += blockDim.x) {
      int r = multi[q];
      lab[r] = lab2[r];
      nrj[r] = nrj2[r];
    }
    __syncthreads();
  }
  for (int q = threadIdx.x; q < M; q += blockDim.x) {
    int r = multi[q];
    int h = rid[lab[r]];
    hr[r] = h;
    succ[r] = nr[r] == h ? -1 : nr[r];
    val[r] = re[r] - rs[r] + 1;
    ishead[r] = h == r;
  }
  __syncthreads();
  for (int it = 0; it < rounds && M > 0; it++) {
    for (int q = threadIdx.x; q < M; q += blockDim.x) {
      int r = multi[q];
      int sc = succ[r];
      val2[r] = val[r] + (sc >= 0 ? val[sc] : 0);
      succ2[r] = sc >= 0 ? succ[sc] : -1;
    }
    __syncthreads();
    for (int q = threadIdx.x; q < M; q += blockDim.x) {
      int r = multi[q];
      val[r] = val2[r];
      succ[r] = succ2[r];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) *valout = val;
}

__global__ void k_rb_cycles2(const int *__restrict__ ishead, const int *__restrict__ cidx,
                             long long *const *__restrict__ valp, const int *__restrict__ rs,
                             const int *__restrict__ lvl, const LevelDesc *__restrict__ lev,
                             const int *__restrict__ R_dev, int *__restrict__ clen,
                             int *__restrict__ clev) {
  CASL_PDL_ENTRY();
  const int R = *R_dev;
  const long long *val = *valp;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < R; r += gridDim.x * blockDim.x) {
    if (!ishead[r]) continue;
    int c = cidx[r];
    clen[c] = (int)val[r];
    clev[c] = lev[lvl[rs[r]]].levt;
  }
}

__global__ void k_rb_gather2(const double *__restrict__ xq, const double *__restrict__ yq, int npt,
                             const int *__restrict__ rid, const int *__restrict__ rs,
                             const int *__restrict__ hr, const int *__restrict__ cidx,
                             long long *const *__restrict__ valp, const int *__restrict__ cst,
                             const int *__restrict__ clen, double *__restrict__ xw,
                             double *__restrict__ yw, int *__restrict__ cidw) {
  CASL_PDL_ENTRY();
  const long long *val = *valp;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npt; i += gridDim.x * blockDim.x) {
    int r = rid[i];
    int c = cidx[hr[r]];
    long long off = (long long)clen[c] - val[r];
    long long pos = cst[c] + off + (i - rs[r]);
    xw[pos] = xq[i];
    yw[pos] = yq[i];
    cidw[pos] = c;
  }
}

// Write the renoded contours back into the node and contour arrays
// (contours.f90:645-680) using the counts left in device memory.
__global__ void k_rb_writeback(const int *__restrict__ cnt, long long npm, long long nm,
                               const int *__restrict__ ocs, const int *__restrict__ olen,
                               const int *__restrict__ olev, const double *__restrict__ xo,
                               const double *__restrict__ yo, double *__restrict__ xq,
                               double *__restrict__ yq, int *__restrict__ nextq,
                               int *__restrict__ i1q, int *__restrict__ i2q,
                               int *__restrict__ npq, int *__restrict__ indq,
                               Scalars *__restrict__ s) {
  CASL_PDL_ENTRY();
  const int nq = cnt[0], npt = cnt[1];
  if (cnt[2] || npt > npm || nq > nm) {
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicExch(&s->error, CASL_ECAPACITY);
    return;
  }
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nq; j += gridDim.x * blockDim.x) {
    i1q[j] = ocs[j];
    i2q[j] = ocs[j] + olen[j] - 1;
    npq[j] = olen[j];
    indq[j] = olev[j];
  }
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npt; i += gridDim.x * blockDim.x) {
    xq[i] = xo[i];
    yq[i] = yo[i];
    int j = contour_of(ocs, nq, i);
    nextq[i] = i + 1 < ocs[j] + olen[j] ? i + 1 : ocs[j];
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    s->nq = nq;
    s->nptq = npt;
  }
}

static inline int gs(long long work) {
  long long g = (work + 255) / 256;
  if (g < 1) g = 1;
  if (g > 148 * 16) g = 148 * 16;
  return (int)g;
}

// Walk-ordered contours of the current link array + renode + write back.
// Issues no host synchronisation: every count stays in device memory and
// every buffer is sized from the node count npt.
static int rebuild_and_renode(casl_handle *h, Arena &ar, int npt, const int *lvl,
                              const LevelDesc *dlev) {
  cudaStream_t st = h->stream;
  int *stf = ar.get<int>(npt), *brk = ar.get<int>(npt), *sx = ar.get<int>(npt);
  int *rid = ar.get<int>(npt), *tmpi = ar.get<int>(scan_tmp_elems(npt) + 4);
  int *dtot = ar.get<int>(8);
  // run arrays (R <= npt)
  int *rs = ar.get<int>(npt), *re = ar.get<int>(npt), *nr = ar.get<int>(npt);
  int *lab = ar.get<int>(npt), *lab2 = ar.get<int>(npt), *nrj = ar.get<int>(npt);
  int *nrj2 = ar.get<int>(npt), *hr = ar.get<int>(npt), *succ = ar.get<int>(npt);
  int *succ2 = ar.get<int>(npt), *ishead = ar.get<int>(npt), *cidx = ar.get<int>(npt);
  long long *val = ar.get<long long>(npt), *val2 = ar.get<long long>(npt);
  long long **valp = ar.get<long long *>(1);
  int *multi = ar.get<int>(npt);
  // cycles (C <= R <= npt)
  int *clen = ar.get<int>(npt), *clev = ar.get<int>(npt), *cst = ar.get<int>(npt);
  double *xw = ar.get<double>(npt), *yw = ar.get<double>(npt);
  int *ocs = ar.get<int>(npt), *olen = ar.get<int>(npt), *olev = ar.get<int>(npt);
  int *cnt = ar.get<int>(4);
  int *nmulti = ar.get<int>(4);
  if (ar.failed) return CASL_ENOMEM;
  const int g = gs(npt);
  CASL_K(k_rb_flags, g, 256, 0, st)(h->nextq, npt, stf, brk);
  exclusive_scan<int>(st, stf, sx, npt, tmpi, dtot);           // dtot[0] = R
  CASL_K(k_rb_runs, g, 256, 0, st)(stf, brk, sx, npt, rid, rs, re);
  {
    const FillJob z[3] = {{ishead, npt, 0u}, {clen, npt, 0u}, {nmulti, 1, 0u}};
    if (int rc = fill_words(st, z, 3)) return rc;
  }
  CASL_K(k_rb_cycles_pre, g, 256, 0, st)(h->nextq, rid, rs, re, dtot, nr, lab, nrj, hr, val, val2,
                                         ishead, multi, nmulti);
  CASL_K(k_rb_cycles_block, 1, 1024, 0, st)(h->nextq, rid, rs, re, dtot, nr, lab, lab2, nrj, nrj2,
                                            hr, succ, succ2, val, val2, ishead, multi, valp,
                                            nmulti);
  exclusive_scan<int>(st, ishead, cidx, npt, tmpi, dtot + 1);  // dtot[1] = C
  CASL_K(k_rb_cycles2, g, 256, 0, st)(ishead, cidx, valp, rs, lvl, dlev, dtot, clen, clev);
  exclusive_scan<int>(st, clen, cst, npt, tmpi, dtot + 2);
  int *cidw = ar.get<int>(npt);
  if (ar.failed) return CASL_ENOMEM;
  CASL_K(k_rb_gather2, g, 256, 0, st)(h->xq, h->yq, npt, rid, rs, hr, cidx, valp, cst, clen, xw, yw,
                                      cidw);
  int rc = check_launch(h);
  if (rc) return rc;
  RenodeIn in{xw, yw, cst, clen, clev, npt, npt, dtot + 1, cidw};
  RenodeOut out{};
  out.xo = h->xqi;  // node-sized scratch of the RK step, free between steps
  out.yo = h->yqi;
  out.ocs = ocs; out.olen = olen; out.olev = olev;
  out.cap = h->npm;
  out.d_counts = cnt;
  rc = renode_batch(h, ar, in, out, RENODE_SURGERY);
  if (rc) return rc;
  CASL_K(k_rb_writeback, gs(h->npm < (1 << 24) ? h->npm : (1 << 24)), 256, 0, st)(
      cnt, h->npm, h->nm, ocs, olen, olev, h->xqi, h->yqi, h->xq, h->yq, h->nextq, h->i1q,
      h->i2q, h->npq, h->indq, h->scal);
  return check_launch(h);
}

int surgery_dev(casl_handle *h) {
  if (h->nq == 0 || h->nptq == 0) return CASL_OK;
  cudaStream_t st = h->stream;
  const Consts &c = h->c;
  const int nq = h->nq, npt = h->nptq;
  const long long nbox_cap = 2LL * npt + nq + 64;
  const long long ne_cap = 16LL * npt + 64;
  size_t need = (size_t)npt * 760 + (size_t)nq * 96 + (size_t)nbox_cap * 24 +
                (size_t)ne_cap * 16 + ((size_t)64 << 20);
  int rc = ensure_scratch(h, need);
  if (rc) return rc;
  Arena ar{(char *)h->sx, h->sx_bytes, 0};
  int *err = &h->scal->error;
  Trace tr;
  tr.begin(st, "start");
  // levels and boxes, on the device
  int *lex = ar.get<int>(nq);
  LevelDesc *dlev = ar.get<LevelDesc>(nq);
  // [0] nlev, [1] nbox, [2] ne, [3] nsurg, [4] box segment entries, [5] box nodes
  int *dtot = ar.get<int>(16);
  int *endnext = ar.get<int>(npt), *lvl = ar.get<int>(npt);
  double *dx = ar.get<double>(npt), *dy = ar.get<double>(npt), *dsq = ar.get<double>(npt);
  double *x0 = ar.get<double>(npt), *y0 = ar.get<double>(npt);
  double *dx0 = ar.get<double>(npt), *dy0 = ar.get<double>(npt);
  int *nq0 = ar.get<int>(npt), *prev0 = ar.get<int>(npt);
  unsigned char *pending = ar.get<unsigned char>(npt + 16);
  unsigned int *wsum = ar.get<unsigned int>((npt >> 14) + 2);
  int *ecount = ar.get<int>(npt), *eoff = ar.get<int>(npt), *nbox_of = ar.get<int>(npt);
  int *bcnt = ar.get<int>(nbox_cap), *kb1 = ar.get<int>(nbox_cap), *cursor = ar.get<int>(nbox_cap);
  int *nbcnt = ar.get<int>(nbox_cap), *nb1 = ar.get<int>(nbox_cap), *nbnode = ar.get<int>(npt);
  int *ncursor = ar.get<int>(nbox_cap), *bbase = ar.get<int>(148 * 16 + 1);
  int *ebox = ar.get<int>(ne_cap), *eib = ar.get<int>(ne_cap), *bnode = ar.get<int>(ne_cap);
  int *bnq = ar.get<int>(ne_cap);
  if (ar.failed) return CASL_ENOMEM;
  const int g = gs(npt), gb = gs(nbox_cap);
  {
    const FillJob z[5] = {{endnext, npt, 0xffffffffu},
                          {bcnt, nbox_cap, 0u},
                          {nbcnt, nbox_cap, 0u},
                          {wsum, (npt >> 14) + 2, 0u},
                          {dtot + 2, 4, 0u}};
    if (int rc = fill_words(st, z, 5)) return rc;
  }
  CASL_K(k_lv_all, 1, SCAN_BLOCK, 0, st)(h->i1q, h->i2q, h->indq, nq, npt, c, dlev, lex, endnext,
                                         dtot, nbox_cap, err);
  CASL_K(k_sg_init, g, 256, 0, st)(h->xq, h->yq, h->nextq, endnext, npt, dx, dy, dsq, x0, y0, dx0,
                                   dy0, nq0, prev0, pending, dlev, dtot, lvl, c, err);
  SurgState S{};
  S.xq = h->xq; S.yq = h->yq; S.dx = dx; S.dy = dy; S.dsq = dsq; S.nextq = h->nextq;
  S.x0 = x0; S.y0 = y0; S.dx0 = dx0; S.dy0 = dy0; S.nq0 = nq0; S.prev0 = prev0; S.lvl = lvl;
  S.pending = pending;
  S.wsum = wsum;
  // count_entries: at most 148*16 blocks, each a whole number of 256-node steps
  const int echunk = (int)((((long long)npt + g - 1) / g + 255) / 256 * 256);
  const int eg = (int)(((long long)npt + echunk - 1) / echunk);
  CASL_K(k_sg_count_entries, eg, 256, 0, st)(S, dlev, npt, echunk, ecount, eoff, bbase, dtot + 2,
                                             nbox_of, nbcnt, c);
  CASL_K(k_sg_emit, g, 256, 0, st)(S, dlev, npt, eoff, bbase, echunk, ecount, ne_cap, ebox, eib,
                                   bcnt, c, err);
  {
    // boxes in 296 chunks (two blocks of 1024 per SM), each a whole number
    // of 1024-box steps
    const long long bchunk = ((nbox_cap + 295) / 296 + 1023) / 1024 * 1024;
    const int bg = (int)((nbox_cap + bchunk - 1) / bchunk);
    CASL_K(k_sg_box_alloc, bg, 1024, 0, st)(bcnt, nbcnt, dtot + 1, nbox_cap, bchunk, kb1, cursor,
                                            nb1, ncursor, dtot + 4);
  }
  CASL_K(k_sg_place, gs(ne_cap), 256, 0, st)(ebox, eib, dtot + 2, ne_cap, cursor, nq0, bnode, bnq);
  CASL_K(k_sg_place_nodes, g, 256, 0, st)(nbox_of, npt, ncursor, nbnode);
  S.kb1 = kb1; S.bcnt = bcnt; S.bnode = bnode; S.bnq = bnq; S.nb1 = nb1; S.nbcnt = nbcnt; S.nbnode = nbnode;
  tr.point("binning");
  CASL_K(k_sg_candidates, g, 256, 0, st)(S, dlev, npt, nbox_of, c);
  tr.point("candidates");
  int *stats = tr.on ? ar.get<int>(2 * (size_t)nq) : nullptr;
  if (stats) CASL_CUDA_TRY(cudaMemsetAsync(stats, 0, 2 * (size_t)nq * sizeof(int), st));
  CASL_K(k_sg_replay, (nq * 32 + 127) / 128, 128, 0, st)(S, dlev, dtot + 0, c, dtot + 3, stats);
  rc = check_launch(h);
  if (rc) return rc;
  tr.point("replay");
  if (stats) {
    std::vector<int> hs(2 * (size_t)nq);
    int nlev = 0;
    CASL_CUDA_TRY(cudaMemcpyAsync(hs.data(), stats, hs.size() * sizeof(int), cudaMemcpyDeviceToHost, st));
    CASL_CUDA_TRY(cudaMemcpyAsync(&nlev, dtot, sizeof(int), cudaMemcpyDeviceToHost, st));
    CASL_CUDA_TRY(cudaStreamSynchronize(st));
    long long sp = 0, ss = 0;
    int mp = 0, ms = 0, wl = 0;
    for (int l = 0; l < nlev; l++) {
      sp += hs[2 * l];
      ss += hs[2 * l + 1];
      if (hs[2 * l] > mp) { mp = hs[2 * l]; wl = l; }
      ms = std::max(ms, hs[2 * l + 1]);
    }
    fprintf(stderr, "[casl trace] replay: %d levels, pending %lld (max %d at level %d, %d surgeries there), surgeries %lld (max %d)\n",
            nlev, sp, mp, wl, hs[2 * wl + 1], ss, ms);
  }
  rc = rebuild_and_renode(h, ar, npt, lvl, dlev);
  if (rc) return rc;
  tr.point("rebuild+renode");
  tr.flush("surgery");
  // the host copies of the counts are refreshed at the next synchronisation
  return CASL_OK;
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
  if (hc[2]) return CASL_ECAPACITY;
  *npr = hc[1];
  if (hc[1] > 0) {
    CASL_CUDA_TRY(cudaMemcpyAsync(xr, xo, hc[1] * sizeof(double), cudaMemcpyDeviceToHost, st));
    CASL_CUDA_TRY(cudaMemcpyAsync(yr, yo, hc[1] * sizeof(double), cudaMemcpyDeviceToHost, st));
    CASL_CUDA_TRY(cudaStreamSynchronize(st));
  }
  return check_launch(h);
}

}  // namespace casl
