// Recontouring (congen.f90:24-441) on the GPU.
//
// 1. Ultra-fine field (16x): contour PV from integer jump counts
//    (con2ugrid, congen.f90:338-441) plus the bilinear residual
//    (congen.f90:45-61), or the bilinear field alone when there are no
//    contours (congen.f90:63-95).
// 2. Every grid-line crossing of every level is enumerated in the
//    reference's numbering order (x lines: ix outer / iy inner, then y lines:
//    iy outer / ix inner, congen.f90:200-254), then stably sorted by level.
// 3. The per-box crossing tables (noctab/icrtab) become a hash on
//    (level, box).  A crossing's successor is the out-crossing of the box it
//    enters; only boxes with two out-crossings (saddles) depend on the order
//    of the reference's traversal, so those few are resolved by a short
//    exact simulation of that traversal over chains.
// 4. Each contour starts at its lowest-numbered crossing (the reference's
//    `free` loop); contours are ordered by level then by that crossing,
//    gathered into walk order and renoded three times (congen.f90:295-310).
// With beta != 0 the PV is not periodic in y and recontouring follows
// econgen.f90 (the reference's ecaps build) instead: the level range and the
// rows iymin..iymax that it needs come from the field's row extremes, the
// rows outside the basic box are its periodic images offset by beta*Ly per
// box, crossings are enumerated over that extended grid in econgen's order,
// and of the traced contours only one periodic image each is kept, its y
// folded back into the box, before the renodes.
#include <cub/device/device_radix_sort.cuh>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include <algorithm>
#include <vector>

#include "renode.cuh"
#include "scan.cuh"
#include "state.cuh"

namespace casl {

// ---------------------------------------------------------------------------
// Ultra-fine field
// ---------------------------------------------------------------------------
__global__ void k_u_scatter(const double *__restrict__ xq, const double *__restrict__ yq,
                            const int *__restrict__ nextq, int npt, double qjump,
                            int *__restrict__ J, int *__restrict__ ljx, Consts c,
                            int *__restrict__ err) {
  CASL_PDL_ENTRY();
  const int nxu = c.nxu, nyu = c.nyu;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npt; i += gridDim.x * blockDim.x) {
    int ia = nextq[i];
    if (ia < 0 || ia >= npt) { atomicExch(err, CASL_EINVAL); continue; }
    double xi = xq[i], yi = yq[i], xa = xq[ia], ya = yq[ia];
    if (!(xi >= c.xmin && xi < c.xmax && yi >= c.ymin && yi < c.ymax)) {
      atomicExch(err, CASL_EDOMAIN);
      continue;
    }
    int ixci = f_int(c.glxui * (xi - c.xmin));
    int ixca = f_int(c.glxui * (xa - c.xmin));
    double xx = xa - xi;
    double dx = xx - c.ellx * f_dint(xx * c.hlxi);
    double yy = ya - yi;
    double dy = yy - c.elly * f_dint(yy * c.hlyi);
    int ixdif = ixca - ixci;
    int nxc = ixdif - nxu * ((2 * ixdif) / nxu);
    if (fabs(yy) > c.hly) {
      double cc = f_sign1(dy);
      double p = -(yi - c.hly * cc) / (dy + c.small);
      int ix = 1 + f_int(c.glxui * fmod(c.ellx + c.hlx + xi + p * dx, c.ellx));
      ix = ix < 1 ? 1 : (ix > nxu ? nxu : ix);
      red_add_s32(&ljx[ix - 1], -(int)cc);
    }
    if (nxc != 0 && nxc >= -nxu && nxc <= nxu) {
      int jump = f_isign1(nxc);
      int ixbeg = ixci + (1 + jump) / 2 + nxu;
      for (int ncr = 0; ncr != nxc; ncr += jump) {
        int m = (ixbeg + ncr) % nxu;
        if (m < 0) m += nxu;
        int ix = 1 + m;
        double xgu = c.xmin + c.glxu * (double)(ix - 1);
        double x2 = xgu - xi;
        double px0 = (x2 - c.ellx * f_dint(x2 * c.hlxi)) / dx;
        double y2 = yi + px0 * dy;
        int iy = 2 + f_int(c.glyui * (y2 - c.elly * f_dint(y2 * c.hlyi) - c.ymin));
        if (iy >= 2 && iy <= nyu) red_add_s32(&J[(long long)(ix - 1) * nyu + (iy - 1)], jump);
      }
    }
  }
}

__global__ void k_u_lbot(const int *__restrict__ ljx, int *__restrict__ J, int nxu, int nyu) {
  CASL_PDL_ENTRY();
  __shared__ int warp_tot[32];
  __shared__ int carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int base = 0; base < nxu; base += blockDim.x) {
    int i = base + threadIdx.x;
    int v = i < nxu ? ljx[i] : 0;
    int x = warp_incl_scan(v);
    if (lane == 31) warp_tot[wid] = x;
    __syncthreads();
    if (wid == 0) {
      int t = lane < nw ? warp_tot[lane] : 0;
      t = warp_incl_scan(t);
      if (lane < nw) warp_tot[lane] = t;
    }
    __syncthreads();
    int incl = x + (wid > 0 ? warp_tot[wid - 1] : 0) + carry;
    if (i < nxu) J[(long long)i * nyu] = incl - v;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry = incl;
    __syncthreads();
  }
}

// column sweep (congen.f90:419-423) with the column sums for the mean
__global__ void k_u_colscan(int *__restrict__ J, int nxu, int nyu,
                            unsigned long long *__restrict__ total) {
  CASL_PDL_ENTRY();
  int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (warp >= nxu) return;
  int *col = J + (long long)warp * nyu;
  int carry = 0;
  long long s = 0;
  for (int base = 0; base < nyu; base += 32) {
    int x = warp_incl_scan(col[base + lane]) + carry;
    col[base + lane] = x;
    s += x;
    carry = __shfl_sync(0xffffffffu, x, 31);
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if (lane == 0) atomicAdd(total, (unsigned long long)s);
}

struct LevInfo {
  int levbeg, levend;
  double qjump, qoff, qjumpi;
};

__device__ __forceinline__ double qtmp_of(int lev, const LevInfo &li) {
  return ((double)lev - 0.5) * li.qjump - li.qoff;
}

// Largest level l whose contour value qtmp(l) = (l - 1/2) qjump - qoff is
// <= v.  qtmp is increasing in l (also as rounded), so an edge with end
// values lo < hi crosses exactly the levels c(lo) < l <= c(hi): those where
// the reference's sign(qa - qtmp) differs at the two ends (congen.f90:205-212).
__device__ __forceinline__ int level_index(double v, const LevInfo &li) {
  int l = (int)floor((v + li.qoff) * li.qjumpi + 0.5);
  while (qtmp_of(l + 1, li) <= v) l++;
  while (qtmp_of(l, li) > v) l--;
  return l;
}

// level_index with the exact checks only near a level boundary: the
// estimate x = (v + qoff)/qjump + 1/2 carries a rounding error of a few
// units of 1e-16 relative (x is at most 65536 + nlevm), as do the qtmp
// values, so a fractional part of x farther than 1e-6 from 0 and 1 fixes
// the level; anything else (and a non-finite v) takes level_index's steps.
__device__ __forceinline__ int level_index_fast(double v, const LevInfo &li) {
  const double x = (v + li.qoff) * li.qjumpi + 0.5;
  const double fl = floor(x), fr = x - fl;
  int l = (int)fl;
  if (fr > 1.0e-6 && fr < 1.0 - 1.0e-6) return l;
  while (qtmp_of(l + 1, li) <= v) l++;
  while (qtmp_of(l, li) > v) l--;
  return l;
}

// One element of the ultra-fine field: (L*qjump - qavg) + bilinear residual,
// or the bilinear residual alone; (ixf, iyf) is the point's 1-based place in
// its coarse cell, q00..q11 the cell's corner values.  Per element the
// expression and its order are the reference's (congen.f90:45-61 on
// con2ugrid's field).  The field kernel and the crossing geometry both
// evaluate the field here, so the crossing positions are computed from the
// very values the crossings were found on.
__device__ __forceinline__ double ufield_elem(int lv, int ixf, int iyf, double q00, double q10,
                                              double q01, double q11, double qjump, double qavg,
                                              int have_contours) {
  const double fac = 1.0 / 16.0;
  const double pxf = fac * (double)(ixf - 1), pxc = 1.0 - pxf;
  const double pyf = fac * (double)(iyf - 1), pyc = 1.0 - pyf;
  const double w00 = pyc * pxc, w10 = pyf * pxc, w01 = pyc * pxf, w11 = pyf * pxf;
  if (have_contours) {
    double v = (double)lv * qjump - qavg;
    return v + w00 * q00 + w10 * q10 + w01 * q01 + w11 * q11;
  }
  return w00 * q00 + w10 * q10 + w01 * q01 + w11 * q11;
}
__device__ __forceinline__ double ufield_qavg(const unsigned long long *lsum, double qjump,
                                              int have_contours, int nxu, int nyu) {
  return have_contours ? qjump * ((double)(long long)(*lsum) / ((double)nxu * (double)nyu)) : 0.0;
}
// the field at the 1-based ultra-fine point (ix, iy)
struct UField {
  const int *L;
  const unsigned long long *lsum;
  const double *qq;
  double qjump;
  int have;
  double bnc;  // beta != 0 without contours: beta*ygu(iy) is added (econgen.f90:94-110)
};
__device__ __forceinline__ double ufield_at(const UField &u, double qavg, int ix, int iy,
                                            const Consts &c) {
  const int n = c.nx;
  const int ixx = (ix - 1) / 16, iyy = (iy - 1) / 16;
  const int ix0 = 1 + ixx, ix1 = 2 + ixx - n * (ix0 / n), ixf = ix - 16 * ixx;
  const int iy0 = 1 + iyy, iy1 = 2 + iyy - n * (iy0 / n), iyf = iy - 16 * iyy;
  const double q00 = u.qq[(long long)(ix0 - 1) * n + iy0 - 1];
  const double q10 = u.qq[(long long)(ix0 - 1) * n + iy1 - 1];
  const double q01 = u.qq[(long long)(ix1 - 1) * n + iy0 - 1];
  const double q11 = u.qq[(long long)(ix1 - 1) * n + iy1 - 1];
  const int lv = u.have ? u.L[(long long)(ix - 1) * c.nyu + iy - 1] : 0;
  const double v = ufield_elem(lv, ixf, iyf, q00, q10, q01, q11, u.qjump, qavg, u.have);
  return u.bnc != 0.0 ? v + u.bnc * (c.ymin + c.glyu * (double)(iy - 1)) : v;
}

// The ultra-fine field, one thread per run of 16 rows of a column: the run
// lies in one coarse cell in y, so the four coarse values are gathered once;
// the levels come in as 16-byte vectors.  Out go the field itself (qa, when
// asked for) and/or its level code lc = level_index(v) clipped to
// [0, 65535], with the field's extremes.  qtmp depends only on qjump and
// nlevm, so the code is known before the level range is.
__global__ void __launch_bounds__(256, 4) k_u_field(const int *__restrict__ L, const unsigned long long *__restrict__ lsum,
                          const double *__restrict__ qq, double qjump, int have_contours,
                          LevInfo lq, double *__restrict__ qa, unsigned short *__restrict__ lc,
                          double *__restrict__ part, Consts c, double bnc) {
  CASL_PDL_ENTRY();
  const int nxu = c.nxu, nyu = c.nyu, n = c.nx;
  const long long nruns = (long long)nxu * (nyu / 16);
  const double qavg = ufield_qavg(lsum, qjump, have_contours, nxu, nyu);
  double mx = -1.0e308, mn = 1.0e308;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nruns;
       t += (long long)gridDim.x * blockDim.x) {
    const int iyy = (int)(t % (nyu / 16)), ix = (int)(t / (nyu / 16)) + 1;
    const int ixx = (ix - 1) / 16;
    const int ix0 = 1 + ixx, ix1 = 2 + ixx - n * (ix0 / n), ixf = ix - 16 * ixx;
    const int iy0 = 1 + iyy, iy1 = 2 + iyy - n * (iy0 / n);
    const double q00 = qq[(long long)(ix0 - 1) * n + iy0 - 1], q10 = qq[(long long)(ix0 - 1) * n + iy1 - 1];
    const double q01 = qq[(long long)(ix1 - 1) * n + iy0 - 1], q11 = qq[(long long)(ix1 - 1) * n + iy1 - 1];
    const long long base = (long long)(ix - 1) * nyu + 16LL * iyy;
    // the run in two halves of 8 points (fewer live registers)
#pragma unroll 1
    for (int hf = 0; hf < 2; hf++) {
      int lv[8];
      if (have_contours) {
        const int4 *l4 = reinterpret_cast<const int4 *>(L + base) + 2 * hf;
        const int4 q0 = l4[0], q1 = l4[1];
        lv[0] = q0.x; lv[1] = q0.y; lv[2] = q0.z; lv[3] = q0.w;
        lv[4] = q1.x; lv[5] = q1.y; lv[6] = q1.z; lv[7] = q1.w;
      } else {
#pragma unroll
        for (int k = 0; k < 8; k++) lv[k] = 0;
      }
      unsigned int code[4];
#pragma unroll
      for (int k = 0; k < 4; k++) {
        double out[2];
#pragma unroll
        for (int h = 0; h < 2; h++) {
          const int iyf = 8 * hf + 2 * k + h;  // 0-based place in the run
          double v = ufield_elem(lv[2 * k + h], ixf, iyf + 1, q00, q10, q01, q11, qjump, qavg,
                                 have_contours);
          if (bnc != 0.0) v = v + bnc * (c.ymin + c.glyu * (double)(16 * iyy + iyf));
          out[h] = v;
          mx = fmax(mx, v);
          mn = fmin(mn, v);
        }
        if (qa) reinterpret_cast<double2 *>(qa + base)[4 * hf + k] = make_double2(out[0], out[1]);
        if (lc) {
          const unsigned int c0 = (unsigned int)min(max(level_index_fast(out[0], lq), 0), 65535);
          const unsigned int c1 = (unsigned int)min(max(level_index_fast(out[1], lq), 0), 65535);
          code[k] = c0 | (c1 << 16);
        }
      }
      if (lc)
        reinterpret_cast<uint4 *>(lc + base)[hf] = make_uint4(code[0], code[1], code[2], code[3]);
    }
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

// ---------------------------------------------------------------------------
// Crossings
// ---------------------------------------------------------------------------
constexpr int EDGES_PER_THREAD = 16;

// Crossings are counted and emitted per chunk of 16 consecutive edges in the
// reference's numbering: x-line edges (ix, iy)-(ix, iy+1) are numbered
// e = ix*nyu + iy, y-line edges (ix, iy)-(ix+1, iy) e = NE + iy*nxu + ix.
// One CTA takes two tiles of CB = 16 columns x RB = 64 rows of level codes,
// each staged in shared memory with the next row and column (periodic):
// each column's 64 codes are 8 16-byte loads, so a tile with its halo is one
// load per thread of its half of the CTA.  An edge whose ends have codes
// ca, cb crosses exactly the levels min(ca, cb) < l <= max(ca, cb) (none
// when they are equal, which takes in equal end values).  Each thread owns
// one chunk of its tile (64 chunks of 16 rows of a column, then 64 chunks of
// 16 columns of a row) and walks its 17 codes: COUNT writes the chunk's
// number of crossings, EMIT writes its crossings (edge, level) from the
// chunk's offset on, edge by edge and level by level, which is the
// reference's order within a chunk.
constexpr int CR_CB = 16, CR_RB = 64;

template <bool EMIT>
__global__ void __launch_bounds__(256) k_cr_tile(const unsigned short *__restrict__ lc, LevInfo li,
                                                 int nxu, int nyu, int *__restrict__ cnt,
                                                 const int *__restrict__ off,
                                                 unsigned long long *__restrict__ redge,
                                                 int *__restrict__ rlev) {
  CASL_PDL_ENTRY();
  __shared__ int Cl[2][CR_CB + 1][CR_RB + 1];  // row length 65
  const int half = threadIdx.x >> 7, t = threadIdx.x & 127;
  const int ntx = nxu / CR_CB, nty = nyu / CR_RB;
  const long long tile = 2LL * blockIdx.x + half;
  const bool live = tile < (long long)ntx * nty;
  const int ix0 = live ? (int)(tile % ntx) * CR_CB : 0, iy0 = live ? (int)(tile / ntx) * CR_RB : 0;
  int(*C)[CR_RB + 1] = Cl[half];
  if (live) {
    for (int q = t; q < (CR_CB + 1) * 9; q += 128) {
      if (q < (CR_CB + 1) * 8) {  // 17 columns x 8 vectors of 8 codes
        const int cc = q >> 3, part = q & 7;
        int ix = ix0 + cc;
        if (ix >= nxu) ix -= nxu;
        const uint4 v = *reinterpret_cast<const uint4 *>(lc + (long long)ix * nyu + iy0 + 8 * part);
        const unsigned int w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int j = 0; j < 4; j++) {
          C[cc][8 * part + 2 * j] = (int)(w[j] & 0xffffu);
          C[cc][8 * part + 2 * j + 1] = (int)(w[j] >> 16);
        }
      } else {  // the row after the tile, periodic
        const int cc = q - (CR_CB + 1) * 8;
        int ix = ix0 + cc, iy = iy0 + CR_RB;
        if (ix >= nxu) ix -= nxu;
        if (iy >= nyu) iy -= nyu;
        C[cc][CR_RB] = lc[(long long)ix * nyu + iy];
      }
    }
  }
  __syncthreads();
  if (!live) return;
  const long long NE = (long long)nxu * nyu;
  // chunk t: x-line chunks 0..63 (column t>>2, rows 16*(t&3)...), then
  // y-line chunks 64..127 (row t-64, columns 0..15)
  const bool xl = t < 64;
  const int cc0 = xl ? t >> 2 : 0, r0 = xl ? 16 * (t & 3) : t - 64;
  const long long e0 = xl ? (long long)(ix0 + cc0) * nyu + (iy0 + r0)
                          : NE + (long long)(iy0 + r0) * nxu + ix0;
  const long long chunk_id = e0 / EDGES_PER_THREAD;
  int pos = EMIT ? off[chunk_id] : 0, total = 0;
  int ca = xl ? C[cc0][r0] : C[0][r0];
#pragma unroll 4
  for (int i = 0; i < 16; i++) {
    const int cb = xl ? C[cc0][r0 + i + 1] : C[i + 1][r0];
    const int l1 = max(min(ca, cb) + 1, li.levbeg), l2 = min(max(ca, cb), li.levend);
    if (!EMIT) {
      total += l2 >= l1 ? l2 - l1 + 1 : 0;
    } else {
      for (int l = l1; l <= l2; l++) {
        redge[pos] = (unsigned long long)(e0 + i);
        rlev[pos] = l - li.levbeg;
        pos++;
      }
    }
    ca = cb;
  }
  if (!EMIT) cnt[chunk_id] = total;
}

// Position and box transitions of every crossing (congen.f90:211-252).
// The end values are the ultra-fine field recomputed at the edge's two
// points, bit for bit the values the level codes were taken from.
__global__ void k_cr_geom(UField uf, const unsigned long long *__restrict__ redge,
                          const int *__restrict__ rlev, long long ncr, LevInfo li, Consts c,
                          double *__restrict__ xcr, double *__restrict__ ycr,
                          unsigned int *__restrict__ kib, unsigned int *__restrict__ kob) {
  CASL_PDL_ENTRY();
  const int nxu = c.nxu, nyu = c.nyu;
  const long long NE = (long long)nxu * nyu;
  const double qavg = ufield_qavg(uf.lsum, uf.qjump, uf.have, nxu, nyu);
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < ncr;
       r += (long long)gridDim.x * blockDim.x) {
    long long e = (long long)redge[r];
    double qtmp = qtmp_of(rlev[r] + li.levbeg, li);
    if (e < NE) {
      int ix = (int)(e / nyu) + 1, iy = (int)(e % nyu) + 1;
      double q0 = ufield_at(uf, qavg, ix, iy, c) - qtmp;
      double q1 = ufield_at(uf, qavg, ix, iy == nyu ? 1 : iy + 1, c) - qtmp;
      int isy = (int)f_sign1(q0);
      int inc = (1 - isy) / 2;
      long long kaa = (long long)(iy - 1) * nxu + 1;
      int j1 = ix + inc, j2 = ix + 1 - inc;
      long long bx1 = j1 == 1 ? nxu - 1 : j1 - 2, bx2 = j2 == 1 ? nxu - 1 : j2 - 2;
      kib[r] = (unsigned int)(kaa + bx1);
      kob[r] = (unsigned int)(kaa + bx2);
      xcr[r] = c.xmin + c.glxu * (double)(ix - 1);
      double ygu = c.ymin + c.glyu * (double)(iy - 1);
      double yy = ygu - c.glyu * q0 / (q1 - q0);
      ycr[r] = c.oms * (yy - c.elly * f_dint(yy * c.hlyi));
    } else {
      long long f = e - NE;
      int iy = (int)(f / nxu) + 1, ix = (int)(f % nxu) + 1;
      double q0 = ufield_at(uf, qavg, ix, iy, c) - qtmp;
      double q1 = ufield_at(uf, qavg, ix == nxu ? 1 : ix + 1, iy, c) - qtmp;
      int isx = (int)f_sign1(q0);
      int inc = (1 - isx) / 2;
      int j1 = iy + 1 - inc, j2 = iy + inc;
      long long by1 = j1 == 1 ? nyu - 1 : j1 - 2, by2 = j2 == 1 ? nyu - 1 : j2 - 2;
      kib[r] = (unsigned int)((long long)nxu * by1 + ix);
      kob[r] = (unsigned int)((long long)nxu * by2 + ix);
      ycr[r] = c.ymin + c.glyu * (double)(iy - 1);
      double xgu = c.xmin + c.glxu * (double)(ix - 1);
      double xx = xgu - c.glxu * q0 / (q1 - q0);
      xcr[r] = c.oms * (xx - c.ellx * f_dint(xx * c.hlxi));
    }
  }
}

// ---------------------------------------------------------------------------
// beta != 0 (econgen.f90:27-488): the grid extended in y
// ---------------------------------------------------------------------------
// PV on a beta-plane is not periodic in y: the periodic image of row iy0 one
// box up carries an extra beta*Ly.  The field is extended over rows
// iymin..iymax, row iy taking the values of basic row iy0 = 1 + mod(iy-1,
// nyu) plus bfac*(iy - iy0), bfac = beta*glyu; contours are traced on the
// extended grid and only one periodic image of each is kept.
struct ExtGrid {
  int iymin, iymax, nby;       // nby: boxes below the basic one (econgen.f90:217)
  double bfac;
  const unsigned short *lc;    // basic rows' level codes, [ix][iy]
  const unsigned short *lcb;   // rows iymin..0, [ix][iy - iymin]
  const unsigned short *lca;   // rows nyu+1..iymax, [ix][iy - nyu - 1]
};
__device__ __forceinline__ int ext_row0(const ExtGrid &g, int iy, int nyu) {
  return iy < 1 ? 1 + (g.nby * nyu + iy - 1) % nyu : (iy > nyu ? 1 + (iy - 1) % nyu : iy);
}
// level code of the 1-based point (ix, iy) of the extended grid
__device__ __forceinline__ int ext_code(const ExtGrid &g, int ix, int iy, int nyu) {
  if (iy < 1) return g.lcb[(long long)(ix - 1) * (1 - g.iymin) + (iy - g.iymin)];
  if (iy > nyu) return g.lca[(long long)(ix - 1) * (g.iymax - nyu) + (iy - nyu - 1)];
  return g.lc[(long long)(ix - 1) * nyu + iy - 1];
}

// Minimum and maximum of the field along every basic row (econgen.f90:
// 114-129): one block per 16 rows, threads over the columns.
__global__ void __launch_bounds__(256) k_u_rowmm(UField uf, Consts c, double *__restrict__ rmin,
                                                 double *__restrict__ rmax) {
  CASL_PDL_ENTRY();
  const int nxu = c.nxu, nyu = c.nyu;
  const double qavg = ufield_qavg(uf.lsum, uf.qjump, uf.have, nxu, nyu);
  const int r0 = 16 * blockIdx.x;
  double mn[16], mx[16];
#pragma unroll
  for (int k = 0; k < 16; k++) {
    mn[k] = 1.0e308;
    mx[k] = -1.0e308;
  }
  for (int ix = threadIdx.x + 1; ix <= nxu; ix += blockDim.x) {
#pragma unroll
    for (int k = 0; k < 16; k++) {
      const double v = ufield_at(uf, qavg, ix, r0 + k + 1, c);
      mn[k] = fmin(mn[k], v);
      mx[k] = fmax(mx[k], v);
    }
  }
  __shared__ double smn[8][16], smx[8][16];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < 16; k++) {
    double a = mn[k], b = mx[k];
    for (int o = 16; o > 0; o >>= 1) {
      a = fmin(a, __shfl_xor_sync(0xffffffffu, a, o));
      b = fmax(b, __shfl_xor_sync(0xffffffffu, b, o));
    }
    if (lane == 0) {
      smn[w][k] = a;
      smx[w][k] = b;
    }
  }
  __syncthreads();
  if (threadIdx.x < 16 && r0 + threadIdx.x < nyu) {
    double a = smn[0][threadIdx.x], b = smx[0][threadIdx.x];
    for (int q = 1; q < (int)(blockDim.x >> 5); q++) {
      a = fmin(a, smn[q][threadIdx.x]);
      b = fmax(b, smx[q][threadIdx.x]);
    }
    rmin[r0 + threadIdx.x] = a;
    rmax[r0 + threadIdx.x] = b;
  }
}

// Level codes of the extension rows: the level index of qa(iy0) +
// bfac*(iy - iy0), the value rounded once as the reference's x-line scan
// forms it (econgen.f90:247-258).
__global__ void k_u_ext(UField uf, ExtGrid g, LevInfo li, Consts c, unsigned short *__restrict__ lcb,
                        unsigned short *__restrict__ lca) {
  CASL_PDL_ENTRY();
  const int nxu = c.nxu, nyu = c.nyu;
  const int nb = 1 - g.iymin, na = g.iymax - nyu, nr = nb + na;
  const double qavg = ufield_qavg(uf.lsum, uf.qjump, uf.have, nxu, nyu);
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < (long long)nxu * nr;
       t += (long long)gridDim.x * blockDim.x) {
    const int ix = (int)(t / nr) + 1, r = (int)(t % nr);
    const int iy = r < nb ? g.iymin + r : nyu + 1 + (r - nb);
    const int iy0 = ext_row0(g, iy, nyu);
    const double v = ufield_at(uf, qavg, ix, iy0, c) + g.bfac * (double)(iy - iy0);
    const unsigned short code = (unsigned short)min(max(level_index(v, li), 0), 65535);
    if (r < nb) lcb[(long long)(ix - 1) * nb + r] = code;
    else lca[(long long)(ix - 1) * na + (r - nb)] = code;
  }
}

// Crossings of the extended grid, counted or emitted per chunk of 16 edges
// in the reference's numbering (econgen.f90:238-348): x-line edges (ix, iy)
// -(ix, iy+1) for iy = iymin..iymax-1, e = (ix-1)(nye-1) + iy - iymin; then
// y-line edges (ix, iy)-(ix+1, iy) for iy = iymin+1..iymax-1,
// e = NEX + (iy-iymin-1) nxu + ix-1.  An edge crosses the levels between its
// ends' codes (the y lines of the extension use the same once-rounded
// values; the reference adds (offset - qtmp) there, which can differ from
// them only when qa lies within an ulp of a level).
template <bool EMIT>
__global__ void k_cre(ExtGrid g, LevInfo li, int nxu, int nyu, long long nedge, long long nex,
                      int *__restrict__ cnt, const int *__restrict__ off,
                      unsigned long long *__restrict__ redge, int *__restrict__ rlev) {
  CASL_PDL_ENTRY();
  const int nye = g.iymax - g.iymin + 1;
  const long long nchunks = (nedge + EDGES_PER_THREAD - 1) / EDGES_PER_THREAD;
  for (long long ch = blockIdx.x * (long long)blockDim.x + threadIdx.x; ch < nchunks;
       ch += (long long)gridDim.x * blockDim.x) {
    const long long e0 = ch * EDGES_PER_THREAD;
    const long long e1 = e0 + EDGES_PER_THREAD < nedge ? e0 + EDGES_PER_THREAD : nedge;
    int pos = EMIT ? off[ch] : 0, total = 0;
    for (long long e = e0; e < e1; e++) {
      int ca, cb;
      if (e < nex) {
        const int ix = (int)(e / (nye - 1)) + 1, iy = g.iymin + (int)(e % (nye - 1));
        ca = ext_code(g, ix, iy, nyu);
        cb = ext_code(g, ix, iy + 1, nyu);
      } else {
        const long long f = e - nex;
        const int iy = g.iymin + 1 + (int)(f / nxu), ix = (int)(f % nxu) + 1;
        ca = ext_code(g, ix, iy, nyu);
        cb = ext_code(g, ix == nxu ? 1 : ix + 1, iy, nyu);
      }
      const int l1 = max(min(ca, cb) + 1, li.levbeg), l2 = min(max(ca, cb), li.levend);
      if (!EMIT) {
        total += l2 >= l1 ? l2 - l1 + 1 : 0;
      } else {
        for (int l = l1; l <= l2; l++) {
          redge[pos] = (unsigned long long)e;
          rlev[pos] = l - li.levbeg;
          pos++;
        }
      }
    }
    if (!EMIT) cnt[ch] = total;
  }
}

// Position and box transitions of every crossing of the extended grid
// (econgen.f90:238-348): y is not folded here; boxes are numbered over the
// extended grid, row by row from iymin (1-based, as the reference's).
__global__ void k_cre_geom(UField uf, ExtGrid g, const unsigned long long *__restrict__ redge,
                           const int *__restrict__ rlev, long long ncr, long long nex, LevInfo li,
                           Consts c, double *__restrict__ xcr, double *__restrict__ ycr,
                           unsigned int *__restrict__ kib, unsigned int *__restrict__ kob) {
  CASL_PDL_ENTRY();
  const int nxu = c.nxu, nyu = c.nyu, nye = g.iymax - g.iymin + 1;
  const double qavg = ufield_qavg(uf.lsum, uf.qjump, uf.have, nxu, nyu);
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < ncr;
       r += (long long)gridDim.x * blockDim.x) {
    const long long e = (long long)redge[r];
    const double qtmp = qtmp_of(rlev[r] + li.levbeg, li);
    if (e < nex) {
      const int ix = (int)(e / (nye - 1)) + 1, iy = g.iymin + (int)(e % (nye - 1));
      double q[2];
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int yy = iy + h, y0 = ext_row0(g, yy, nyu);
        const double v = (yy >= 1 && yy <= nyu)
                             ? ufield_at(uf, qavg, ix, yy, c)
                             : ufield_at(uf, qavg, ix, y0, c) + g.bfac * (double)(yy - y0);
        q[h] = v - qtmp;
      }
      const int isy = (int)f_sign1(q[0]);
      const int inc = (1 - isy) / 2;
      const long long kaa = (long long)(iy - g.iymin) * nxu + 1;
      const int j1 = ix + inc, j2 = ix + 1 - inc;
      const long long bx1 = j1 == 1 ? nxu - 1 : j1 - 2, bx2 = j2 == 1 ? nxu - 1 : j2 - 2;
      kib[r] = (unsigned int)(kaa + bx1);
      kob[r] = (unsigned int)(kaa + bx2);
      xcr[r] = c.xmin + c.glxu * (double)(ix - 1);
      ycr[r] = (c.glyu * (double)(iy - 1) + c.ymin) - c.glyu * q[0] / (q[1] - q[0]);
    } else {
      const long long f = e - nex;
      const int iy = g.iymin + 1 + (int)(f / nxu), ix = (int)(f % nxu) + 1;
      const int y0 = ext_row0(g, iy, nyu);
      const bool basic = iy >= 1 && iy <= nyu;
      const double qadd = g.bfac * (double)(iy - y0) - qtmp;
      double q[2];
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int xx = h == 0 ? ix : (ix == nxu ? 1 : ix + 1);
        q[h] = basic ? ufield_at(uf, qavg, xx, iy, c) - qtmp : ufield_at(uf, qavg, xx, y0, c) + qadd;
      }
      const int isx = (int)f_sign1(q[0]);
      const int inc = (1 - isx) / 2;
      const long long kaa = (long long)(iy - 1 - g.iymin) * nxu + ix;
      kib[r] = (unsigned int)(kaa + (long long)(1 - inc) * nxu);
      kob[r] = (unsigned int)(kaa + (long long)inc * nxu);
      ycr[r] = c.glyu * (double)(iy - 1) + c.ymin;
      const double xgu = c.xmin + c.glxu * (double)(ix - 1);
      const double xx = xgu - c.glxu * q[0] / (q[1] - q[0]);
      xcr[r] = c.oms * (xx - c.ellx * f_dint(xx * c.hlxi));
    }
  }
}

// One periodic image per contour (econgen.f90:238-246): bit 0 of flags[k]
// is set when a crossing of contour k lies below ymin, bit 1 when one lies
// below ymax; k is kept when bit 0 is clear and bit 1 set.
__global__ void k_ec_flags(const double *__restrict__ yw, const int *__restrict__ cidw, long long N,
                           Consts c, int *__restrict__ flags) {
  CASL_PDL_ENTRY();
  for (long long w = blockIdx.x * (long long)blockDim.x + threadIdx.x; w < N;
       w += (long long)gridDim.x * blockDim.x) {
    const double y = yw[w];
    const int f = (y < c.ymin ? 1 : 0) | (y < c.ymax ? 2 : 0);
    if (f) atomicOr(&flags[cidw[w]], f);
  }
}
__global__ void k_ec_keep(const int *__restrict__ flags, const int *__restrict__ clen, int C,
                          int *__restrict__ klen, int *__restrict__ kone) {
  CASL_PDL_ENTRY();
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < C; k += gridDim.x * blockDim.x) {
    const bool keep = !(flags[k] & 1) && (flags[k] & 2);
    klen[k] = keep ? clen[k] : 0;
    kone[k] = keep ? 1 : 0;
  }
}
// The kept contours' crossings, y folded into [ymin, ymax) by
// mod(y + yoff, elly) + ymin (econgen.f90:249-252), and their contour list.
__global__ void k_ec_compact(const double *__restrict__ xw, const double *__restrict__ yw,
                             const int *__restrict__ cidw, long long N, const int *__restrict__ coff,
                             const int *__restrict__ klen, const int *__restrict__ koff,
                             const int *__restrict__ kidx, Consts c, double yoff,
                             double *__restrict__ xw2, double *__restrict__ yw2,
                             int *__restrict__ cidw2) {
  CASL_PDL_ENTRY();
  for (long long w = blockIdx.x * (long long)blockDim.x + threadIdx.x; w < N;
       w += (long long)gridDim.x * blockDim.x) {
    const int k = cidw[w];
    if (!klen[k]) continue;
    const long long d = koff[k] + (w - coff[k]);
    xw2[d] = xw[w];
    yw2[d] = fmod(yw[w] + yoff, c.elly) + c.ymin;
    cidw2[d] = kidx[k];
  }
}
__global__ void k_ec_contours(const int *__restrict__ clen, const int *__restrict__ clevt, int C,
                              const int *__restrict__ klen, const int *__restrict__ koff,
                              const int *__restrict__ kidx, int *__restrict__ cs2,
                              int *__restrict__ len2, int *__restrict__ lev2) {
  CASL_PDL_ENTRY();
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < C; k += gridDim.x * blockDim.x) {
    if (!klen[k]) continue;
    const int j = kidx[k];
    cs2[j] = koff[k];
    len2[j] = clen[k];
    lev2[j] = clevt[k];
  }
}

// ---------------------------------------------------------------------------
// (level, box) -> out-crossings hash (the reference's noctab/icrtab)
// ---------------------------------------------------------------------------
constexpr unsigned long long HEMPTY = ~0ull;

__device__ __forceinline__ unsigned long long hkey(int lev, unsigned int box) {
  return ((unsigned long long)(unsigned int)lev << 32) | box;
}
__device__ __forceinline__ unsigned long long hmix(unsigned long long k) {
  k ^= k >> 33;
  k *= 0xff51afd7ed558ccdULL;
  k ^= k >> 33;
  k *= 0xc4ceb9fe1a85ec53ULL;
  k ^= k >> 33;
  return k;
}

// One bucket per (level, box) key: the key and its (at most two) out-
// crossings share 16 bytes, so a probe touches one sector.  The two slots
// are filled in arrival order; readers that need them ordered take min/max.
struct __align__(16) HBucket {
  unsigned long long key;
  int s0, s1;
};

// Crossings [0, n) of a batch of consecutive levels; slots store the global
// crossing index base + r.
__global__ void k_h_insert(const int *__restrict__ rlev, const unsigned int *__restrict__ kob,
                           long long n, int base, HBucket *__restrict__ hb,
                           unsigned long long mask, int *__restrict__ err) {
  CASL_PDL_ENTRY();
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < n;
       r += (long long)gridDim.x * blockDim.x) {
    unsigned long long k = hkey(rlev[r], kob[r]);
    unsigned long long p = hmix(k) & mask;
    const int slot = base + (int)r;
    bool inserted = false;
    for (unsigned long long probe = 0; probe <= mask; probe++) {
      unsigned long long prev = atomicCAS(&hb[p].key, HEMPTY, k);
      if (prev == HEMPTY || prev == k) {
        if (atomicCAS(&hb[p].s0, -1, slot) != -1)
          if (atomicCAS(&hb[p].s1, -1, slot) != -1) atomicExch(err, CASL_ECAPACITY);
        inserted = true;
        break;
      }
      p = (p + 1) & mask;
    }
    // a full table would leave this crossing out of the (level, box) table
    if (!inserted) atomicExch(err, CASL_ECAPACITY);
  }
}

// Successor of each crossing of the batch.  A crossing that enters a saddle
// box (two out-crossings) gets succ = -1 and, in sadslot, the box's two
// out-crossings packed as (lower << 32) | higher: the pair names the box
// once the table has been reused for the next batch.  -1 elsewhere.
__global__ void k_h_succ(const int *__restrict__ rlev, const unsigned int *__restrict__ kib,
                         long long n, const HBucket *__restrict__ hb, unsigned long long mask,
                         int *__restrict__ succ, long long *__restrict__ sadslot,
                         int *__restrict__ err) {
  CASL_PDL_ENTRY();
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < n;
       r += (long long)gridDim.x * blockDim.x) {
    const unsigned long long k = hkey(rlev[r], kib[r]);
    unsigned long long p = hmix(k) & mask;
    bool found = false;
    HBucket v;
    for (unsigned long long probe = 0; probe <= mask; probe++) {
      v = hb[p];
      if (v.key == k) {
        found = true;
        break;
      }
      if (v.key == HEMPTY) break;
      p = (p + 1) & mask;
    }
    if (!found) {
      atomicExch(err, CASL_EINVAL);
      succ[r] = -1;
      sadslot[r] = -1;
      continue;
    }
    if (v.s1 < 0) {
      succ[r] = v.s0;
      sadslot[r] = -1;
    } else {
      succ[r] = -1;
      sadslot[r] = (long long)(((unsigned long long)min(v.s0, v.s1) << 32) |
                               (unsigned int)max(v.s0, v.s1));
    }
  }
}

// first crossing of each level (crossings are sorted by level); lstart[nlev] = n
__global__ void k_lev_starts(const int *__restrict__ rlev, long long n, int nlev,
                             long long *__restrict__ lstart) {
  CASL_PDL_ENTRY();
  for (int l = blockIdx.x * blockDim.x + threadIdx.x; l <= nlev; l += gridDim.x * blockDim.x) {
    long long lo = 0, hi = n;
    while (lo < hi) {
      const long long mid = (lo + hi) >> 1;
      if (rlev[mid] < l) lo = mid + 1; else hi = mid;
    }
    lstart[l] = lo;
  }
}

// contour start flags and lengths for plain cycles (start = cycle minimum)
__global__ void k_ct_plain(const int *__restrict__ lab, const int *__restrict__ term,
                           const int *__restrict__ val, long long ncr, int *__restrict__ startf,
                           int *__restrict__ clenr) {
  CASL_PDL_ENTRY();
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < ncr;
       r += (long long)gridDim.x * blockDim.x) {
    bool st = !term[r] && lab[r] == (int)r;
    startf[r] = st;
    clenr[r] = st ? val[r] : 0;
  }
}

// A crossing in walk layout: its position and contour in one 32-byte record,
// so that the scattered store of each crossing fills one whole sector (a
// partial sector costs a read of the sector as well); k_walk_split then
// turns the records into the walk arrays with coalesced accesses.
struct __align__(32) WalkRec {
  double x, y;
  int cid, pad[3];
};
__device__ __forceinline__ void put_rec(WalkRec *__restrict__ rec, long long pos, double x,
                                        double y, int cid) {
  double2 *p = reinterpret_cast<double2 *>(rec + pos);
  p[0] = make_double2(x, y);
  reinterpret_cast<int4 *>(p + 1)[0] = make_int4(cid, 0, 0, 0);
}
__global__ void k_walk_split(const WalkRec *__restrict__ rec, long long ncr,
                             double *__restrict__ xw, double *__restrict__ yw,
                             int *__restrict__ cidw) {
  CASL_PDL_ENTRY();
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < ncr;
       p += (long long)gridDim.x * blockDim.x) {
    const double2 v = reinterpret_cast<const double2 *>(rec + p)[0];
    xw[p] = v.x;
    yw[p] = v.y;
    cidw[p] = rec[p].cid;  // the contour of every walk position, for the first renode
  }
}

// positions of plain-cycle crossings in walk layout
__global__ void k_ct_gather_plain(const int *__restrict__ lab, const int *__restrict__ term,
                                  const int *__restrict__ val, const int *__restrict__ cidx,
                                  const int *__restrict__ coff, const int *__restrict__ clen,
                                  const double *__restrict__ xcr, const double *__restrict__ ycr,
                                  long long ncr, WalkRec *__restrict__ rec) {
  CASL_PDL_ENTRY();
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < ncr;
       r += (long long)gridDim.x * blockDim.x) {
    if (term[r]) continue;
    int s = lab[r];
    int c = cidx[s];
    long long pos = (long long)coff[c] + (clen[c] - val[r]);
    put_rec(rec, pos, xcr[r], ycr[r], c);
  }
}

// chain crossings: position from the per-chain placement of the simulation
__global__ void k_ct_gather_chain(const int *__restrict__ term, const int *__restrict__ ep,
                                  const int *__restrict__ val, const int *__restrict__ chain_of_end,
                                  const long long *__restrict__ chpos, const int *__restrict__ chlen,
                                  const int *__restrict__ chrot, const int *__restrict__ chclen,
                                  const int *__restrict__ chcont, const double *__restrict__ xcr,
                                  const double *__restrict__ ycr, long long ncr,
                                  WalkRec *__restrict__ rec) {
  CASL_PDL_ENTRY();
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < ncr;
       r += (long long)gridDim.x * blockDim.x) {
    if (!term[r]) continue;
    int ch = chain_of_end[ep[r]];
    if (ch < 0) continue;
    int local = chlen[ch] - val[r];          // position from the chain start
    long long pos;
    int rot = chrot[ch];
    if (rot < 0) {
      pos = chpos[ch] + local;
    } else {
      // first chain of a contour started mid-chain at local index rot
      int L = chclen[ch];
      int rel = local >= rot ? local - rot : L - rot + local;
      pos = chpos[ch] + rel;
    }
    put_rec(rec, pos, xcr[r], ycr[r], chcont[ch]);
  }
}

__global__ void k_lev_of_contour(const int *__restrict__ startf, const int *__restrict__ rlev,
                                 const int *__restrict__ cidx, long long ncr, LevInfo li,
                                 int nlevm, int *__restrict__ clevt) {
  CASL_PDL_ENTRY();
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < ncr;
       r += (long long)gridDim.x * blockDim.x) {
    if (!startf[r]) continue;
    int lev = rlev[r] + li.levbeg;
    clevt[cidx[r]] = lev - nlevm + (lev - 1) / nlevm - 1;
  }
}

__global__ void k_set_counts2(Scalars *s, const int *cnt) {
  CASL_PDL_ENTRY();
  s->nq = cnt[0];
  s->nptq = cnt[1];
}
__global__ void k_out_contours(const int *__restrict__ ocs, const int *__restrict__ olen,
                               const int *__restrict__ olev, int nq, int *__restrict__ i1q,
                               int *__restrict__ i2q, int *__restrict__ npq,
                               int *__restrict__ indq) {
  CASL_PDL_ENTRY();
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nq; j += gridDim.x * blockDim.x) {
    i1q[j] = ocs[j];
    i2q[j] = ocs[j] + olen[j] - 1;
    npq[j] = olen[j];
    indq[j] = olev[j];
  }
}
__global__ void k_out_links(const int *__restrict__ ocs, const int *__restrict__ olen, int nq,
                            int npt, int *__restrict__ nextq) {
  CASL_PDL_ENTRY();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npt; i += gridDim.x * blockDim.x) {
    int j = contour_of(ocs, nq, i);
    nextq[i] = i + 1 < ocs[j] + olen[j] ? i + 1 : ocs[j];
  }
}


// ---------------------------------------------------------------------------
// List ranking of the crossing successor graph with splitters.
// Splitters: every K-th crossing and every chain start (a crossing no one
// points to); each walks its segment up to the next splitter.  Cycles that
// hold no sampled crossing get every crossing as a splitter in a second
// round.  Pointer jumping then runs on the (few) splitters only, and the
// result expands back to: term (on a chain), lab (cycle minimum / chain
// minimum at chain starts), val (cycles: crossings from here to the end of
// the walk that starts at the cycle minimum; chains: to the chain end,
// inclusive) and ep (chain end).
// ---------------------------------------------------------------------------
__global__ void k_sp_pred(const int *__restrict__ succ, long long N, int *__restrict__ pred) {
  CASL_PDL_ENTRY();
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < N;
       r += (long long)gridDim.x * blockDim.x) {
    int s = succ[r];
    if (s >= 0) pred[s] = (int)r;
  }
}
// A walk step reads the next node's successor and splitter flag (sf, one
// 8-byte load) and writes the node's (owner, offset) pair (own, one 8-byte
// store): two random accesses per step.  isspl keeps the flags as a plain
// array for the scan.  The sampled crossings are those whose index hashes
// to 0 mod K, not every K-th index: along a contour the indices often step
// by a constant (parallel contours put the same number of crossings in
// every row), and an arithmetic sample can then miss a whole contour.  All
// splitters (sampled ones and chain starts) are appended to xlist, so the
// walks run one thread per splitter with no idle lanes.
__device__ __forceinline__ unsigned int sp_hash(unsigned int x) {
  x ^= x >> 16;
  x *= 0x7feb352dU;
  x ^= x >> 15;
  x *= 0x846ca68bU;
  x ^= x >> 16;
  return x;
}
// Appends go through one atomic per block and tile of the crossings: the
// block's flags are counted by ballots, so the list keeps index order within
// a block.
__device__ __forceinline__ void sp_append(bool f, int r, int *__restrict__ xlist,
                                          int *__restrict__ nx, int *wtot, int *wbase) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const unsigned m = __ballot_sync(0xffffffffu, f);
  if (lane == 0) wtot[w] = __popc(m);
  __syncthreads();
  if (threadIdx.x == 0) {
    int t = 0;
    for (int i = 0; i < nw; i++) {
      const int c = wtot[i];
      wtot[i] = t;
      t += c;
    }
    *wbase = t ? atomicAdd(nx, t) : 0;
  }
  __syncthreads();
  if (f) xlist[*wbase + wtot[w] + __popc(m & ((1u << lane) - 1))] = r;
  __syncthreads();
}
__global__ void k_sp_flag(const int *__restrict__ pred, const int *__restrict__ succ, long long N,
                          int K, int *__restrict__ isspl, int2 *__restrict__ sf,
                          int2 *__restrict__ own, int *__restrict__ xlist,
                          int *__restrict__ nx) {
  CASL_PDL_ENTRY();
  __shared__ int wtot[32], wbase;
  for (long long b0 = blockIdx.x * (long long)blockDim.x; b0 < N;
       b0 += (long long)gridDim.x * blockDim.x) {
    const long long r = b0 + threadIdx.x;
    int f = 0;
    if (r < N) {
      f = sp_hash((unsigned int)r) % (unsigned int)K == 0 || pred[r] < 0;
      isspl[r] = f;
      sf[r] = make_int2(succ[r], f);
      own[r] = make_int2(-1, 0);
    }
    sp_append(f != 0, (int)r, xlist, nx, wtot, &wbase);
  }
}
// Walks from the splitters xlist[0 .. *nx) up to the next splitter, one
// thread per splitter.  A walk longer than N steps (impossible for a
// successor graph) sets err and ends.
__global__ void k_sp_walk(const int2 *__restrict__ sf, long long N, const int *__restrict__ xlist,
                          const int *__restrict__ nx, int2 *__restrict__ own,
                          int *__restrict__ nexts_c, int *__restrict__ seglen_c,
                          int *__restrict__ segmin_c, int *__restrict__ segend_c,
                          int *__restrict__ err) {
  CASL_PDL_ENTRY();
  const int total = *nx;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
    const int s = xlist[t];
    int v = s, k = 0, mn = s, nxt = -1;
    own[s] = make_int2(s, 0);
    int n = sf[s].x;
    for (long long guard = 0; guard < N; guard++) {
      if (n < 0) { nxt = -1; break; }
      const int2 q = sf[n];  // successor and flag of the next node
      if (q.y) { nxt = n; break; }
      v = n;
      n = q.x;
      k++;
      own[v] = make_int2(s, k);
      mn = min(mn, v);
      if (guard == N - 1) atomicExch(err, CASL_EINVAL);
    }
    nexts_c[s] = nxt;
    seglen_c[s] = k + 1;
    segmin_c[s] = mn;
    segend_c[s] = v;
  }
}
// crossings on cycles that hold no splitter: every one becomes a splitter
// (its walk ends at once, the successor being one too)
__global__ void k_sp_unowned(long long N, const int2 *__restrict__ own, int *__restrict__ isspl,
                             int2 *__restrict__ sf, int *__restrict__ xlist,
                             int *__restrict__ nx) {
  CASL_PDL_ENTRY();
  __shared__ int wtot[32], wbase;
  for (long long b0 = blockIdx.x * (long long)blockDim.x; b0 < N;
       b0 += (long long)gridDim.x * blockDim.x) {
    const long long r = b0 + threadIdx.x;
    bool f = false;
    if (r < N && own[r].x < 0) {
      f = true;
      isspl[r] = 1;
      sf[r].y = 1;
    }
    sp_append(f, (int)r, xlist, nx, wtot, &wbase);
  }
}
__global__ void k_sp_compact(const int *__restrict__ isspl, const int *__restrict__ srank, long long N,
                             const int *__restrict__ nexts_c, const int *__restrict__ seglen_c,
                             const int *__restrict__ segmin_c, const int *__restrict__ segend_c,
                             int *__restrict__ nexts, int *__restrict__ seglen,
                             int *__restrict__ segmin, int *__restrict__ segend) {
  CASL_PDL_ENTRY();
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < N;
       r += (long long)gridDim.x * blockDim.x) {
    if (!isspl[r]) continue;
    int k = srank[r];
    int nx = nexts_c[r];
    nexts[k] = nx < 0 ? -1 : srank[nx];
    seglen[k] = seglen_c[r];
    segmin[k] = segmin_c[r];
    segend[k] = segend_c[r];
  }
}
// Pointer jumping over the splitters.  Each splitter's jump state is one
// 16-byte record (next, minimum, terminal flag, last), so that a round
// gathers two records (at next and at last) instead of four separate words.
__global__ void k_sp_init(const int *__restrict__ nexts, const int *__restrict__ segmin, int S,
                          int4 *__restrict__ J) {
  CASL_PDL_ENTRY();
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < S; k += gridDim.x * blockDim.x) {
    const int n = nexts[k];
    J[k] = make_int4(n < 0 ? k : n, segmin[k], n < 0, n < 0 ? k : n);
  }
}
__global__ void k_sp_jump1(const int4 *__restrict__ J, int S, int4 *__restrict__ J2) {
  CASL_PDL_ENTRY();
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < S; k += gridDim.x * blockDim.x) {
    const int4 a = J[k];
    const int4 b = J[a.x];
    J2[k] = make_int4(b.x, min(a.y, b.y), a.z | b.z, J[a.w].w);
  }
}
// the jump results as the separate arrays the later passes read
__global__ void k_sp_unpack1(const int4 *__restrict__ J, int S, int *__restrict__ mn,
                             int *__restrict__ tm, int *__restrict__ lastp) {
  CASL_PDL_ENTRY();
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < S; k += gridDim.x * blockDim.x) {
    const int4 a = J[k];
    mn[k] = a.y;
    tm[k] = a.z;
    lastp[k] = a.w;
  }
}
// list for suffix sums: cycles are cut before the splitter holding the cycle
// minimum; chains end at their last splitter
// (link, suffix sum) of the suffix-sum jumps, one 16-byte record
struct __align__(16) SlSuf {
  long long suf;
  int sl, pad;
};
__global__ void k_sp_list(const int *__restrict__ nexts, const int *__restrict__ mn,
                          const int *__restrict__ tm, const int2 *__restrict__ own,
                          const int *__restrict__ srank, const int *__restrict__ seglen, int S,
                          SlSuf *__restrict__ L, int *__restrict__ head) {
  CASL_PDL_ENTRY();
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < S; k += gridDim.x * blockDim.x) {
    int n = nexts[k], sl;
    if (tm[k]) {
      sl = n;
      head[k] = -1;
    } else {
      int h = srank[own[mn[k]].x];
      head[k] = h;
      sl = n == h ? -1 : n;
    }
    L[k] = SlSuf{(long long)seglen[k], sl, 0};
  }
}
__global__ void k_sp_jump2(const SlSuf *__restrict__ L, int S, SlSuf *__restrict__ L2) {
  CASL_PDL_ENTRY();
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < S; k += gridDim.x * blockDim.x) {
    const SlSuf a = L[k];
    if (a.sl >= 0) {
      const SlSuf b = L[a.sl];
      L2[k] = SlSuf{a.suf + b.suf, b.sl, 0};
    } else {
      L2[k] = a;
    }
  }
}
__global__ void k_sp_unpack2(const SlSuf *__restrict__ L, int S, long long *__restrict__ suf) {
  CASL_PDL_ENTRY();
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < S; k += gridDim.x * blockDim.x)
    suf[k] = L[k].suf;
}
__global__ void k_sp_expand(long long N, const int2 *__restrict__ own,
                            const int *__restrict__ srank, const int *__restrict__ tm,
                            const int *__restrict__ mn, const long long *__restrict__ suf,
                            const int *__restrict__ head, const int *__restrict__ lastp,
                            const int *__restrict__ segend, int *__restrict__ term,
                            int *__restrict__ lab, int *__restrict__ val, int *__restrict__ ep) {
  CASL_PDL_ENTRY();
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < N;
       c += (long long)gridDim.x * blockDim.x) {
    const int2 oc = own[c];
    int k = srank[oc.x];
    int o = oc.y;
    if (tm[k]) {
      term[c] = 1;
      val[c] = (int)(suf[k] - o);
      ep[c] = segend[lastp[k]];
      lab[c] = o == 0 ? mn[k] : (int)c;
    } else {
      int m = mn[k];
      long long L = suf[head[k]];
      long long pos = (L - suf[k]) + o - own[m].y;
      if (pos < 0) pos += L;
      term[c] = 0;
      val[c] = (int)(L - pos);
      lab[c] = m;
      ep[c] = (int)c;
    }
  }
}

// --- small device helpers for the saddle bookkeeping ------------------------
__global__ void k_sd_endflag(const int *__restrict__ succ, long long ncr, int *__restrict__ flag) {
  CASL_PDL_ENTRY();
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < ncr;
       r += (long long)gridDim.x * blockDim.x)
    flag[r] = succ[r] < 0;
}
__global__ void k_sd_compact(const int *__restrict__ flag, const int *__restrict__ pos,
                             const long long *__restrict__ sadslot, long long ncr,
                             int *__restrict__ oidx, long long *__restrict__ oslot) {
  CASL_PDL_ENTRY();
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < ncr;
       r += (long long)gridDim.x * blockDim.x)
    if (flag[r]) {
      oidx[pos[r]] = (int)r;
      oslot[pos[r]] = sadslot[r];
    }
}
__global__ void k_gather_i(const int *__restrict__ src, const int *__restrict__ idx, int m,
                           int *__restrict__ dst) {
  CASL_PDL_ENTRY();
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x)
    dst[k] = src[idx[k]];
}
// three arrays gathered at the same indices: dst[j*m + k] = src_j[idx[k]]
__global__ void k_gather3_i(const int *__restrict__ s0, const int *__restrict__ s1,
                            const int *__restrict__ s2, const int *__restrict__ idx, int m,
                            int *__restrict__ dst) {
  CASL_PDL_ENTRY();
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x) {
    const int i = idx[k];
    dst[k] = s0[i];
    dst[m + k] = s1[i];
    dst[2 * m + k] = s2[i];
  }
}
__global__ void k_ct_len(const int *__restrict__ startf, const int *__restrict__ clenr,
                         const int *__restrict__ cidx, long long ncr, int *__restrict__ clen) {
  CASL_PDL_ENTRY();
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < ncr;
       r += (long long)gridDim.x * blockDim.x)
    if (startf[r]) clen[cidx[r]] = clenr[r];
}
__global__ void k_chain_of_end(const int *__restrict__ ends, int nch, int *__restrict__ coe) {
  CASL_PDL_ENTRY();
  for (int ch = blockIdx.x * blockDim.x + threadIdx.x; ch < nch; ch += gridDim.x * blockDim.x)
    coe[ends[ch]] = ch;
}
__global__ void k_set_starts(const int *__restrict__ st_idx, const int *__restrict__ st_len, int m,
                             int *__restrict__ startf, int *__restrict__ clenr) {
  CASL_PDL_ENTRY();
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x) {
    startf[st_idx[k]] = 1;
    clenr[st_idx[k]] = st_len[k];
  }
}

static inline int gsz(long long work) {
  long long g = (work + 255) / 256;
  if (g < 1) g = 1;
  if (g > 148 * 32) g = 148 * 32;
  return (int)g;
}

#define RC_TRY(x)        \
  do {                   \
    int _r = (x);        \
    if (_r) return _r;   \
  } while (0)

static int fetch_err(casl_handle *h) {
  int e = 0;
  cudaMemcpyAsync(&e, &h->scal->error, sizeof(int), cudaMemcpyDeviceToHost, h->stream);
  cudaError_t ce = cudaStreamSynchronize(h->stream);
  if (ce != cudaSuccess) return set_cuda_error(h, ce);
  return e;
}

int recontour_dev(casl_handle *h, const double *qq) {
  cudaStream_t st = h->stream;
  const Consts &c = h->c;
  const int nxu = c.nxu, nyu = c.nyu;
  const long long NU = (long long)nxu * nyu;
  const double qjump = h->qjump;
  const int have = h->nptq > 0 && h->nq > 0;
  // beta != 0 recontours as econgen.f90 does (the reference's ecaps build):
  // beta*Ly must be a whole number of contour intervals (econgen.f90:52-60,
  // where the reference stops)
  const bool econ = c.beffect != 0;
  const double bfac = c.beta * c.glyu, ppvdif = c.beta * c.elly;
  if (econ) {
    const double brat = ppvdif * (1.0 / qjump);
    if (!(fabs(brat - (double)llround(brat)) <= 1.0e-7)) return CASL_EINVAL;
  }
  const double bnc = econ && !have ? c.beta : 0.0;
  cudaMemsetAsync(&h->scal->error, 0, sizeof(int), st);
  Trace tr;
  tr.begin(st, "start");
  struct Flush {
    Trace &t;
    ~Flush() { t.flush("recontour"); }
  } flush_at_exit{tr};

  // --- 1. ultra-fine field ---------------------------------------------------
  if (!have && !econ) {
    // l1norm (generic.f90:180-194) of the full field: nothing to contour if ~0
    std::vector<double> hq((size_t)c.nx * c.ny);
    CASL_CUDA_TRY(cudaMemcpyAsync(hq.data(), qq, hq.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    CASL_CUDA_TRY(cudaStreamSynchronize(st));
    double l1 = 0.0;
    for (double v : hq) l1 += fabs(v);
    if (c.garea * l1 < c.small) {
      h->nq = h->nptq = 0;
      h->hscal->nq = h->hscal->nptq = 0;
      int z[2] = {0, 0};
      int *dz = &h->scal->nq;
      CASL_CUDA_TRY(cudaMemcpyAsync(dz, z, 2 * sizeof(int), cudaMemcpyHostToDevice, st));
      CASL_CUDA_TRY(cudaStreamSynchronize(st));
      return CASL_OK;
    }
  }
  // Field memory: level codes + integer levels + per-chunk crossing counts;
  // kept for the whole call.
  const long long nchunks_f = (2 * NU + EDGES_PER_THREAD - 1) / EDGES_PER_THREAD;
  size_t need_field = (size_t)NU * 6 + (size_t)nchunks_f * 8 + (size_t)nxu * 4 +
                      (size_t)nyu * 16 + ((size_t)64 << 20);
  RC_TRY(ensure_scratch(h, need_field));
  Arena ar{(char *)h->sx, h->sx_bytes, 0};
  unsigned short *lc = ar.get<unsigned short>(NU);
  int *Lu = ar.get<int>(NU);
  int *ljx = ar.get<int>(nxu);
  unsigned long long *lsum = ar.get<unsigned long long>(4);
  double *part = ar.get<double>(2 * 4096);
  double *rmn = ar.get<double>(nyu), *rmx = ar.get<double>(nyu);
  int *dtot = ar.get<int>(16);
  if (ar.failed) return CASL_ENOMEM;
  if (have) {
    CASL_CUDA_TRY(cudaMemsetAsync(Lu, 0, (size_t)NU * sizeof(int), st));
    CASL_CUDA_TRY(cudaMemsetAsync(ljx, 0, (size_t)nxu * sizeof(int), st));
    CASL_CUDA_TRY(cudaMemsetAsync(lsum, 0, sizeof(unsigned long long), st));
    tr.point("u_memset");
    CASL_K(k_u_scatter, gsz(h->nptq), 256, 0, st)(h->xq, h->yq, h->nextq, h->nptq, qjump, Lu, ljx, c,
                                              &h->scal->error);
    tr.point("u_scatter");
    CASL_K(k_u_lbot, 1, 1024, 0, st)(ljx, Lu, nxu, nyu);
    CASL_K(k_u_colscan, (nxu * 32 + 255) / 256, 256, 0, st)(Lu, nxu, nyu, lsum);
    tr.point("u_colscan");
  }
  // qtmp(l) = (l - 1/2) qjump - qoff with qoff = qjump*nlevm (congen.f90:156-173)
  LevInfo li;
  li.qjump = qjump;
  li.qjumpi = 1.0 / qjump;
  li.qoff = qjump * (double)h->p.nlevm;
  li.levbeg = li.levend = 0;
  const int fb = 4096;
  CASL_K(k_u_field, fb, 256, 0, st)(Lu, lsum, qq, qjump, have, li, nullptr, lc, part, c, bnc);
  RC_TRY(check_launch(h));
  RC_TRY(fetch_err(h));
  std::vector<double> hp(2 * fb);
  CASL_CUDA_TRY(cudaMemcpyAsync(hp.data(), part, hp.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
  CASL_CUDA_TRY(cudaStreamSynchronize(st));
  double qamax = hp[0], qamin = hp[1];
  for (int b = 1; b < fb; b++) {
    qamax = std::max(qamax, hp[2 * b]);
    qamin = std::min(qamin, hp[2 * b + 1]);
  }
  tr.point("field");
  const UField uf{have ? Lu : nullptr, lsum, qq, qjump, have, bnc};
  // beta != 0: the extent of the y-extended grid (econgen.f90:112-171), on
  // the host from the rows' minima and maxima
  ExtGrid eg{};
  if (econ) {
    CASL_K(k_u_rowmm, nyu / 16, 256, 0, st)(uf, c, rmn, rmx);
    std::vector<double> qqmin(nyu + 2), qqmax(nyu + 2);
    CASL_CUDA_TRY(cudaMemcpyAsync(qqmin.data() + 1, rmn, nyu * sizeof(double), cudaMemcpyDeviceToHost, st));
    CASL_CUDA_TRY(cudaMemcpyAsync(qqmax.data() + 1, rmx, nyu * sizeof(double), cudaMemcpyDeviceToHost, st));
    CASL_CUDA_TRY(cudaStreamSynchronize(st));
    qqmin[nyu + 1] = qqmin[1] + ppvdif;
    qqmax[nyu + 1] = qqmax[1] + ppvdif;
    qamin = qqmin[1];
    qamax = qqmax[1];
    for (int iy = 2; iy <= nyu + 1; iy++) {
      qamin = std::min(qamin, qqmin[iy]);
      qamax = std::max(qamax, qqmax[iy]);
    }
    // the lowest and highest rows that meet a level of the basic box; the
    // reference assumes fewer than 100 periodic boxes
    const int levmin = (int)(qamin * li.qjumpi - 0.5);
    double qlev = ((double)levmin + 0.5) * qjump;
    int iy = 1;
    for (;;) {
      iy = iy - 1;
      if (iy < -100 * nyu) return CASL_ECAPACITY;
      const int iy0 = 1 + (100 * nyu + iy - 1) % nyu;
      if (bfac * (double)(iy - iy0) + qqmax[iy0] <= qlev) break;
    }
    eg.iymin = iy;
    const int levmax = (int)(qamax * li.qjumpi + 0.5);
    qlev = ((double)levmax - 0.5) * qjump;
    iy = nyu + 1;
    for (;;) {
      iy = iy + 1;
      if (iy > 101 * nyu) return CASL_ECAPACITY;
      const int iy0 = 1 + (iy - 1) % nyu;
      if (bfac * (double)(iy - iy0) + qqmin[iy0] >= qlev) break;
    }
    eg.iymax = iy;
    eg.nby = 1 - eg.iymin / nyu;
    eg.bfac = bfac;
    eg.lc = lc;
    // box numbers of the extended grid are 32-bit
    if ((long long)nxu * (eg.iymax - eg.iymin + 2) >= (1LL << 32)) return CASL_ECAPACITY;
  }
  // --- 2. levels (congen.f90:156-173; econgen.f90:131-134) -------------------
  li.levbeg = (int)((li.qoff + qamin) * li.qjumpi + 0.5) + 1;
  li.levend = (int)((li.qoff + qamax) * li.qjumpi + 0.5);
  // the level codes hold 0..65535: levels must lie inside
  if (li.levbeg <= li.levend && (li.levbeg < 1 || li.levend > 65534)) return CASL_ECAPACITY;
  auto set_empty = [&]() -> int {
    h->nq = h->nptq = 0;
    int z[2] = {0, 0};
    CASL_CUDA_TRY(cudaMemcpyAsync(&h->scal->nq, z, 2 * sizeof(int), cudaMemcpyHostToDevice, st));
    CASL_CUDA_TRY(cudaStreamSynchronize(st));
    return CASL_OK;
  };
  if (li.levbeg > li.levend) return set_empty();
  const int nlev = li.levend - li.levbeg + 1;

  tr.point("levels");
  // --- 3. crossings in reference order, stably sorted by level ----------------
  // beta != 0: the extension rows' codes, then the extended grid's edges
  const int nye = econ ? eg.iymax - eg.iymin + 1 : 0;
  const long long nex = econ ? (long long)nxu * (nye - 1) : 0;
  const long long NE2 = econ ? nex + (long long)nxu * (nye - 2) : 2 * NU;
  const long long nchunks = (NE2 + EDGES_PER_THREAD - 1) / EDGES_PER_THREAD;
  int *ccnt, *coffs, *tmpi;
  if (econ) {
    // codes and chunk counts in a buffer of their own (the field arena is
    // sized before the extension is known)
    const int nb = 1 - eg.iymin, na = eg.iymax - nyu;
    const size_t bcodes = ((size_t)nxu * (nb + na) * 2 + 255) / 256 * 256;
    const size_t need = bcodes + (size_t)nchunks * 8 + (size_t)(scan_tmp_elems(nchunks) + 4) * 4 +
                        ((size_t)1 << 20);
    if (h->sxe_bytes < need) {
      if (h->sxe) cudaFree(h->sxe);
      h->sxe = nullptr;
      h->sxe_bytes = 0;
      CASL_CUDA_TRY(cudaMalloc(&h->sxe, need + need / 2));
      h->sxe_bytes = need + need / 2;
    }
    Arena are{(char *)h->sxe, h->sxe_bytes, 0};
    unsigned short *lcb = are.get<unsigned short>((long long)nxu * nb);
    unsigned short *lca = are.get<unsigned short>((long long)nxu * na);
    ccnt = are.get<int>(nchunks);
    coffs = are.get<int>(nchunks);
    tmpi = are.get<int>(scan_tmp_elems(nchunks) + 4);
    if (are.failed) return CASL_ENOMEM;
    eg.lcb = lcb;
    eg.lca = lca;
    CASL_K(k_u_ext, gsz((long long)nxu * (nb + na)), 256, 0, st)(uf, eg, li, c, lcb, lca);
    CASL_K(k_cre<false>, gsz(nchunks), 256, 0, st)(eg, li, nxu, nyu, NE2, nex, ccnt, nullptr,
                                                   nullptr, nullptr);
  } else {
    ccnt = ar.get<int>(nchunks);
    coffs = ar.get<int>(nchunks);
    tmpi = ar.get<int>(scan_tmp_elems(nchunks) + 4);
    if (ar.failed) return CASL_ENOMEM;
  }
  const long long ntile = (long long)(nxu / CR_CB) * (nyu / CR_RB);
  const int tgrid = (int)((ntile + 1) / 2);
  if (!econ)
    CASL_K(k_cr_tile<false>, tgrid, 256, 0, st)(lc, li, nxu, nyu, ccnt, nullptr, nullptr, nullptr);
  tr.point("cr_count");
  exclusive_scan<int>(st, ccnt, coffs, nchunks, tmpi, dtot);
  int ncr_i = 0;
  CASL_CUDA_TRY(cudaMemcpyAsync(&ncr_i, dtot, sizeof(int), cudaMemcpyDeviceToHost, st));
  CASL_CUDA_TRY(cudaStreamSynchronize(st));
  const long long ncr = ncr_i;
  if (tr.on) fprintf(stderr, "[casl trace] recontour: %lld crossings on %d levels\n", ncr, nlev);
  if (ncr == 0) return set_empty();
  // Per-crossing storage lives in a second arena sized from the count, so
  // that the ultra-fine field in the first one is kept.
  int endbit = 1;
  while ((1 << endbit) < nlev + 1) endbit++;
  size_t sort_bytes = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, (int *)nullptr, (int *)nullptr,
                                  (unsigned long long *)nullptr, (unsigned long long *)nullptr,
                                  (int)ncr, 0, endbit, st);
  {
    unsigned long long capb = 1;
    while (capb < (unsigned long long)(2 * ncr)) capb <<= 1;
    long long capn = std::max<long long>(ncr * 2, h->npm);
    size_t need2 = (size_t)ncr * 640 + (size_t)capb * 16 + (size_t)capn * 32 + sort_bytes +
                   ((size_t)64 << 20);
    RC_TRY(ensure_scratch2(h, need2));
  }
  Arena ar2{(char *)h->sx2, h->sx2_bytes, 0};
  unsigned long long *redge = ar2.get<unsigned long long>(ncr), *redge2 = ar2.get<unsigned long long>(ncr);
  int *rlev = ar2.get<int>(ncr), *rlev2 = ar2.get<int>(ncr);
  int *tmpi2 = ar2.get<int>(scan_tmp_elems(ncr) + 4);
  void *sort_tmp = ar2.get<char>(sort_bytes + 16);
  if (ar2.failed) return CASL_ENOMEM;
  tr.point("cr_alloc");
  if (econ)
    CASL_K(k_cre<true>, gsz(nchunks), 256, 0, st)(eg, li, nxu, nyu, NE2, nex, nullptr, coffs,
                                                  redge, rlev);
  else
    CASL_K(k_cr_tile<true>, tgrid, 256, 0, st)(lc, li, nxu, nyu, nullptr, coffs, redge, rlev);
  tr.point("cr_emit");
  CASL_CUDA_TRY(cub::DeviceRadixSort::SortPairs(sort_tmp, sort_bytes, rlev, rlev2, redge, redge2,
                                                (int)ncr, 0, endbit, st));
  std::swap(rlev, rlev2);
  std::swap(redge, redge2);
  tr.point("cr_sort");
  double *xcr = ar2.get<double>(ncr), *ycr = ar2.get<double>(ncr);
  unsigned int *kib = ar2.get<unsigned int>(ncr), *kob = ar2.get<unsigned int>(ncr);
  if (ar2.failed) return CASL_ENOMEM;
  if (econ)
    CASL_K(k_cre_geom, gsz(ncr), 256, 0, st)(uf, eg, redge, rlev, ncr, nex, li, c, xcr, ycr, kib,
                                             kob);
  else
    CASL_K(k_cr_geom, gsz(ncr), 256, 0, st)(uf, redge, rlev, ncr, li, c, xcr, ycr, kib, kob);
  RC_TRY(check_launch(h));

  tr.point("crossings");
  // --- 4. box tables: hash (level, box) -> two out-crossing slots ------------
  // Levels go through the table in batches of about HB_BATCH crossings (2M:
  // a 64 MB table; 1M batches measured 20 % slower), so that the table (16
  // bytes per bucket, load <= 1/2) stays in L2 while the
  // batch's inserts and look-ups run; the keys carry the level, so a batch of
  // several levels shares one table.  CASL_HASH_BATCH=<crossings> overrides
  // the batch size (a test forces one level per batch with it).
  long long HB_BATCH = 1 << 21;
  if (const char *e = getenv("CASL_HASH_BATCH"))
    if (atoll(e) > 0) HB_BATCH = atoll(e);
  long long *lstart = ar2.get<long long>(nlev + 1);
  if (ar2.failed) return CASL_ENOMEM;
  std::vector<long long> hl(nlev + 1);
  CASL_K(k_lev_starts, 1, 128, 0, st)(rlev, ncr, nlev, lstart);
  CASL_CUDA_TRY(cudaMemcpyAsync(hl.data(), lstart, (nlev + 1) * sizeof(long long),
                                cudaMemcpyDeviceToHost, st));
  CASL_CUDA_TRY(cudaStreamSynchronize(st));
  tr.point("hash_levels");
  std::vector<std::pair<long long, long long>> batches;  // [r0, r1)
  for (int l = 0; l < nlev;) {
    int l2 = l + 1;
    while (l2 < nlev && hl[l2 + 1] - hl[l] <= HB_BATCH) l2++;
    batches.push_back({hl[l], hl[l2]});
    l = l2;
  }
  long long bmax = 0;
  for (auto &b : batches) bmax = std::max(bmax, b.second - b.first);
  unsigned long long cap = 1;
  while (cap < (unsigned long long)(2 * bmax)) cap <<= 1;
  HBucket *hb = ar2.get<HBucket>(cap);
  int *succ = ar2.get<int>(ncr);
  long long *sadslot = ar2.get<long long>(ncr);
  if (ar2.failed) return CASL_ENOMEM;
  for (auto &b : batches) {
    const long long nb = b.second - b.first;
    if (nb <= 0) continue;
    unsigned long long cb = 1;
    while (cb < (unsigned long long)(2 * nb)) cb <<= 1;
    CASL_CUDA_TRY(cudaMemsetAsync(hb, 0xff, cb * sizeof(HBucket), st));  // empty key, slots -1
    CASL_K(k_h_insert, gsz(nb), 256, 0, st)(rlev + b.first, kob + b.first, nb, (int)b.first, hb,
                                           cb - 1, &h->scal->error);
    CASL_K(k_h_succ, gsz(nb), 256, 0, st)(rlev + b.first, kib + b.first, nb, hb, cb - 1,
                                         succ + b.first, sadslot + b.first, &h->scal->error);
  }
  RC_TRY(check_launch(h));
  RC_TRY(fetch_err(h));
  if (tr.on)
    fprintf(stderr, "[casl trace] hash: %zu level batches, table %llu buckets\n", batches.size(),
            cap);

  tr.point("hash");
  // --- 5. list ranking over crossings (splitters) ------------------------------
  int *lab = ar2.get<int>(ncr), *term = ar2.get<int>(ncr), *val = ar2.get<int>(ncr),
      *ep = ar2.get<int>(ncr);
  int *pred = ar2.get<int>(ncr), *isspl = ar2.get<int>(ncr), *srank = ar2.get<int>(ncr);
  int2 *sf = ar2.get<int2>(ncr), *own = ar2.get<int2>(ncr);
  int *nexts_c = ar2.get<int>(ncr), *seglen_c = ar2.get<int>(ncr), *segmin_c = ar2.get<int>(ncr),
      *segend_c = ar2.get<int>(ncr);
  if (ar2.failed) return CASL_ENOMEM;
  int g = gsz(ncr);
  CASL_CUDA_TRY(cudaMemsetAsync(pred, 0xff, ncr * sizeof(int), st));
  CASL_K(k_sp_pred, g, 256, 0, st)(succ, ncr, pred);
  tr.point("rk_pred");
  // term and val are written only by the expansion at the end: until then
  // they hold the lists of splitters
  const int K = 16;
  int *xl1 = term, *xl2 = val, *nx1 = dtot + 10, *nx2 = dtot + 11;
  CASL_CUDA_TRY(cudaMemsetAsync(nx1, 0, 2 * sizeof(int), st));
  CASL_K(k_sp_flag, g, 256, 0, st)(pred, succ, ncr, K, isspl, sf, own, xl1, nx1);
  tr.point("rk_flag");
  CASL_K(k_sp_walk, gsz(ncr / K + 1), 256, 0, st)(sf, ncr, xl1, nx1, own, nexts_c, seglen_c,
                                                  segmin_c, segend_c, &h->scal->error);
  tr.point("rk_walk1");
  CASL_K(k_sp_unowned, g, 256, 0, st)(ncr, own, isspl, sf, xl2, nx2);
  CASL_K(k_sp_walk, g, 256, 0, st)(sf, ncr, xl2, nx2, own, nexts_c, seglen_c, segmin_c,
                                   segend_c, &h->scal->error);
  tr.point("rk_walk2");
  exclusive_scan<int>(st, isspl, srank, ncr, tmpi2, dtot + 6);
  int S = 0;
  CASL_CUDA_TRY(cudaMemcpyAsync(&S, dtot + 6, sizeof(int), cudaMemcpyDeviceToHost, st));
  CASL_CUDA_TRY(cudaStreamSynchronize(st));
  if (S <= 0) return CASL_EINVAL;
  int *nexts = ar2.get<int>(S), *seglen = ar2.get<int>(S), *segmin = ar2.get<int>(S),
      *segend = ar2.get<int>(S);
  int *smn = ar2.get<int>(S), *stm = ar2.get<int>(S), *slp = ar2.get<int>(S),
      *shead = ar2.get<int>(S);
  long long *ssuf = ar2.get<long long>(S);
  int4 *jA = ar2.get<int4>(S), *jB = ar2.get<int4>(S);
  SlSuf *lA = ar2.get<SlSuf>(S), *lB = ar2.get<SlSuf>(S);
  if (ar2.failed) return CASL_ENOMEM;
  tr.point("rk_scan");
  CASL_K(k_sp_compact, g, 256, 0, st)(isspl, srank, ncr, nexts_c, seglen_c, segmin_c, segend_c,
                                      nexts, seglen, segmin, segend);
  int gsS = gsz(S);
  int rounds = 1;
  while ((1LL << rounds) < S) rounds++;
  rounds++;
  CASL_K(k_sp_init, gsS, 256, 0, st)(nexts, segmin, S, jA);
  for (int it = 0; it < rounds; it++) {
    CASL_K(k_sp_jump1, gsS, 256, 0, st)(jA, S, jB);
    std::swap(jA, jB);
  }
  CASL_K(k_sp_unpack1, gsS, 256, 0, st)(jA, S, smn, stm, slp);
  CASL_K(k_sp_list, gsS, 256, 0, st)(nexts, smn, stm, own, srank, seglen, S, lA, shead);
  for (int it = 0; it < rounds; it++) {
    CASL_K(k_sp_jump2, gsS, 256, 0, st)(lA, S, lB);
    std::swap(lA, lB);
  }
  CASL_K(k_sp_unpack2, gsS, 256, 0, st)(lA, S, ssuf);
  tr.point("rk_jump");
  CASL_K(k_sp_expand, g, 256, 0, st)(ncr, own, srank, stm, smn, ssuf, shead, slp, segend,
                                     term, lab, val, ep);
  RC_TRY(check_launch(h));
  if (tr.on) {
    std::vector<int> sl(S);
    CASL_CUDA_TRY(cudaMemcpyAsync(sl.data(), seglen, S * sizeof(int), cudaMemcpyDeviceToHost, st));
    CASL_CUDA_TRY(cudaStreamSynchronize(st));
    long long tot = 0;
    int mx = 0;
    for (int x : sl) {
      tot += x;
      mx = std::max(mx, x);
    }
    fprintf(stderr, "[casl trace] ranking: %d splitters, %d jump rounds; segment length mean %.2f, max %d\n",
            S, rounds, (double)tot / S, mx);
  }

  tr.point("rk_expand");
  // --- 6. saddle chains: exact simulation of the reference traversal ----------
  // Only the crossings entering saddle boxes and the chain starts come to the
  // host; everything of size ncr stays on the device.
  int *endflag = ar2.get<int>(ncr), *endpos = ar2.get<int>(ncr);
  if (ar2.failed) return CASL_ENOMEM;
  CASL_K(k_sd_endflag, g, 256, 0, st)(succ, ncr, endflag);
  exclusive_scan<int>(st, endflag, endpos, ncr, tmpi2, dtot + 3);
  int nends = 0;
  CASL_CUDA_TRY(cudaMemcpyAsync(&nends, dtot + 3, sizeof(int), cudaMemcpyDeviceToHost, st));
  CASL_CUDA_TRY(cudaStreamSynchronize(st));
  // gather src[idx[k]] for a host index list
  int *gidx = nullptr, *gout = nullptr;
  long long gcap = 0;
  auto gather = [&](const int *src, const std::vector<int> &idx, std::vector<int> &out) -> int {
    int m = (int)idx.size();
    out.assign(m, 0);
    if (m == 0) return CASL_OK;
    if (m > gcap) {
      gidx = ar2.get<int>(m);
      gout = ar2.get<int>(m);
      gcap = m;
      if (ar2.failed) return CASL_ENOMEM;
    }
    CASL_CUDA_TRY(cudaMemcpyAsync(gidx, idx.data(), m * sizeof(int), cudaMemcpyHostToDevice, st));
    CASL_K(k_gather_i, gsz(m), 256, 0, st)(src, gidx, m, gout);
    CASL_CUDA_TRY(cudaMemcpyAsync(out.data(), gout, m * sizeof(int), cudaMemcpyDeviceToHost, st));
    CASL_CUDA_TRY(cudaStreamSynchronize(st));
    return CASL_OK;
  };
  int nsad_contours = 0;
  std::vector<int> sad_start;      // start crossing of each saddle contour
  std::vector<int> sad_len;        // its length
  std::vector<int> ch_end, ch_len, ch_rot, ch_clen, ch_cont;
  std::vector<long long> ch_pos;   // position relative to the contour start (set later)
  if (nends > 0) {
    int *d_eidx = ar2.get<int>(nends);
    long long *d_eslot = ar2.get<long long>(nends);
    if (ar2.failed) return CASL_ENOMEM;
    CASL_K(k_sd_compact, g, 256, 0, st)(endflag, endpos, sadslot, ncr, d_eidx, d_eslot);
    std::vector<int> eidx(nends);
    std::vector<long long> eslot(nends);
    CASL_CUDA_TRY(cudaMemcpyAsync(eidx.data(), d_eidx, nends * sizeof(int), cudaMemcpyDeviceToHost, st));
    CASL_CUDA_TRY(cudaMemcpyAsync(eslot.data(), d_eslot, nends * sizeof(long long), cudaMemcpyDeviceToHost, st));
    CASL_CUDA_TRY(cudaStreamSynchronize(st));
    std::vector<long long> sad_p(eslot);
    std::sort(sad_p.begin(), sad_p.end());
    sad_p.erase(std::unique(sad_p.begin(), sad_p.end()), sad_p.end());
    int nsb = (int)sad_p.size();
    // each saddle box is named by its two out-crossings, lower index first
    std::vector<int> slot2(2 * nsb);
    for (int b = 0; b < nsb; b++) {
      slot2[2 * b] = (int)((unsigned long long)sad_p[b] >> 32);
      slot2[2 * b + 1] = (int)((unsigned long long)sad_p[b] & 0xffffffffull);
    }
    // chain starts (the saddle out-crossings) and their ends, lengths, minima
    int nch = 2 * nsb;
    std::vector<int> cstart(slot2), cend(nch), clen(nch), cmin(nch);
    {
      // ends, lengths and minima at the chain starts: one gather, one copy
      int *d_idx = ar2.get<int>(nch), *d_out = ar2.get<int>(3LL * nch);
      if (ar2.failed) return CASL_ENOMEM;
      std::vector<int> h_out(3 * (size_t)nch);
      CASL_CUDA_TRY(cudaMemcpyAsync(d_idx, cstart.data(), nch * sizeof(int), cudaMemcpyHostToDevice, st));
      CASL_K(k_gather3_i, gsz(nch), 256, 0, st)(ep, val, lab, d_idx, nch, d_out);
      CASL_CUDA_TRY(cudaMemcpyAsync(h_out.data(), d_out, h_out.size() * sizeof(int), cudaMemcpyDeviceToHost, st));
      CASL_CUDA_TRY(cudaStreamSynchronize(st));
      std::copy(h_out.begin(), h_out.begin() + nch, cend.begin());
      std::copy(h_out.begin() + nch, h_out.begin() + 2 * nch, clen.begin());
      std::copy(h_out.begin() + 2 * nch, h_out.end(), cmin.begin());
    }
    std::vector<int> val_at_min;
    RC_TRY(gather(val, cmin, val_at_min));
    std::vector<std::pair<int, int>> start2ch;
    for (int ch = 0; ch < nch; ch++) start2ch.push_back({cstart[ch], ch});
    std::sort(start2ch.begin(), start2ch.end());
    auto chain_starting_at = [&](int s) -> int {
      auto it = std::lower_bound(start2ch.begin(), start2ch.end(), std::make_pair(s, -1));
      return (it != start2ch.end() && it->first == s) ? it->second : -1;
    };
    // saddle box entered by each chain end
    std::vector<std::pair<int, long long>> end_slot(nends);
    for (int k = 0; k < nends; k++) end_slot[k] = {eidx[k], eslot[k]};
    std::sort(end_slot.begin(), end_slot.end());
    std::vector<int> box_of_end(nch);
    for (int ch = 0; ch < nch; ch++) {
      auto it = std::lower_bound(end_slot.begin(), end_slot.end(), std::make_pair(cend[ch], -1LL));
      if (it == end_slot.end() || it->first != cend[ch]) return CASL_EINVAL;
      box_of_end[ch] = (int)(std::lower_bound(sad_p.begin(), sad_p.end(), it->second) - sad_p.begin());
    }
    std::vector<int> noc(nsb, 2);
    std::vector<char> used(nch, 0);
    ch_end = cend;
    ch_len = clen;
    ch_rot.assign(nch, -1);
    ch_clen.assign(nch, 0);
    ch_cont.assign(nch, -1);
    ch_pos.assign(nch, 0);
    // chains in order of their smallest crossing: contour starts
    std::vector<int> order(nch);
    for (int k = 0; k < nch; k++) order[k] = k;
    std::sort(order.begin(), order.end(), [&](int a, int b) { return cmin[a] < cmin[b]; });
    for (int oc : order) {
      if (used[oc]) continue;
      int icr = cmin[oc];            // the contour's first crossing
      std::vector<int> seq;          // chains in traversal order
      int ch = oc;
      used[ch] = 1;
      seq.push_back(ch);
      int guard = 0;
      while (true) {
        int b = box_of_end[ch];
        int k = noc[b];
        if (k < 1 || k > 2) return CASL_EINVAL;
        int icrn = slot2[2 * b + k - 1];
        if (icrn == icr) break;      // closes at the start (no decrement)
        noc[b] = k - 1;
        int nxt = chain_starting_at(icrn);
        if (nxt < 0) return CASL_EINVAL;
        if (nxt == oc) break;        // back into the first chain, which holds icr
        if (used[nxt]) return CASL_EINVAL;
        used[nxt] = 1;
        seq.push_back(nxt);
        ch = nxt;
        if (++guard > nch + 2) return CASL_EINVAL;
      }
      // lay out: first chain rotated to start at icr, then the others
      int L = 0;
      for (int q : seq) L += clen[q];
      int cont = nsad_contours++;
      sad_start.push_back(icr);
      sad_len.push_back(L);
      int first = seq[0];
      int rot = clen[first] - val_at_min[oc];  // local index of icr in its chain
      ch_rot[first] = rot;
      ch_clen[first] = clen[first];
      ch_cont[first] = cont;
      ch_pos[first] = 0;
      long long off = clen[first] - rot;   // crossings from icr to the chain end
      for (size_t q = 1; q < seq.size(); q++) {
        ch_cont[seq[q]] = cont;
        ch_pos[seq[q]] = off;
        off += clen[seq[q]];
      }
    }
  }

  tr.point("saddles");
  // --- 7. contour order and walk layout ---------------------------------------
  int *startf = ar2.get<int>(ncr), *clenr = ar2.get<int>(ncr), *cidx = ar2.get<int>(ncr);
  if (ar2.failed) return CASL_ENOMEM;
  CASL_K(k_ct_plain, g, 256, 0, st)(lab, term, val, ncr, startf, clenr);
  if (nsad_contours > 0) {
    int *d_si = ar2.get<int>(nsad_contours), *d_sl = ar2.get<int>(nsad_contours);
    if (ar2.failed) return CASL_ENOMEM;
    CASL_CUDA_TRY(cudaMemcpyAsync(d_si, sad_start.data(), nsad_contours * sizeof(int), cudaMemcpyHostToDevice, st));
    CASL_CUDA_TRY(cudaMemcpyAsync(d_sl, sad_len.data(), nsad_contours * sizeof(int), cudaMemcpyHostToDevice, st));
    CASL_K(k_set_starts, gsz(nsad_contours), 256, 0, st)(d_si, d_sl, nsad_contours, startf, clenr);
  }
  exclusive_scan<int>(st, startf, cidx, ncr, tmpi2, dtot + 1);
  int C = 0;
  CASL_CUDA_TRY(cudaMemcpyAsync(&C, dtot + 1, sizeof(int), cudaMemcpyDeviceToHost, st));
  CASL_CUDA_TRY(cudaStreamSynchronize(st));
  if (C == 0) return set_empty();
  int *clen = ar2.get<int>(C), *coff = ar2.get<int>(C), *clevt = ar2.get<int>(C);
  double *xw = ar2.get<double>(ncr), *yw = ar2.get<double>(ncr);
  int *cidw = ar2.get<int>(ncr);
  WalkRec *rec = ar2.get<WalkRec>(ncr);
  if (ar2.failed) return CASL_ENOMEM;
  // contour lengths in contour order, and their offsets
  CASL_K(k_ct_len, g, 256, 0, st)(startf, clenr, cidx, ncr, clen);
  exclusive_scan<int>(st, clen, coff, C, tmpi2, dtot + 2);
  CASL_K(k_ct_gather_plain, g, 256, 0, st)(lab, term, val, cidx, coff, clen, xcr, ycr, ncr, rec);
  int nch = (int)ch_end.size();
  if (nch > 0) {
    // absolute position of every chain; the first chain of a contour is
    // rotated to begin at the contour's first crossing, its head wrapping
    // to the end of the contour
    std::vector<int> sad_cidx, sad_off;
    RC_TRY(gather(cidx, sad_start, sad_cidx));
    RC_TRY(gather(coff, sad_cidx, sad_off));
    std::vector<long long> abs_pos(nch);
    std::vector<int> rotlen(nch, 0), chc(nch);
    for (int ch = 0; ch < nch; ch++) {
      int cont = ch_cont[ch];
      if (cont < 0) return CASL_EINVAL;
      abs_pos[ch] = sad_off[cont] + ch_pos[ch];
      if (ch_rot[ch] >= 0) rotlen[ch] = sad_len[cont];
      chc[ch] = sad_cidx[cont];
    }
    long long *d_pos = ar2.get<long long>(nch);
    int *d_len = ar2.get<int>(nch), *d_rot = ar2.get<int>(nch), *d_cl = ar2.get<int>(nch);
    int *d_ends = ar2.get<int>(nch), *d_cc = ar2.get<int>(nch);
    int *chain_of_end = ar2.get<int>(ncr);
    if (ar2.failed) return CASL_ENOMEM;
    CASL_CUDA_TRY(cudaMemcpyAsync(d_pos, abs_pos.data(), nch * sizeof(long long), cudaMemcpyHostToDevice, st));
    CASL_CUDA_TRY(cudaMemcpyAsync(d_len, ch_len.data(), nch * sizeof(int), cudaMemcpyHostToDevice, st));
    CASL_CUDA_TRY(cudaMemcpyAsync(d_rot, ch_rot.data(), nch * sizeof(int), cudaMemcpyHostToDevice, st));
    CASL_CUDA_TRY(cudaMemcpyAsync(d_cl, rotlen.data(), nch * sizeof(int), cudaMemcpyHostToDevice, st));
    CASL_CUDA_TRY(cudaMemcpyAsync(d_ends, ch_end.data(), nch * sizeof(int), cudaMemcpyHostToDevice, st));
    CASL_CUDA_TRY(cudaMemcpyAsync(d_cc, chc.data(), nch * sizeof(int), cudaMemcpyHostToDevice, st));
    CASL_CUDA_TRY(cudaMemsetAsync(chain_of_end, 0xff, ncr * sizeof(int), st));
    CASL_K(k_chain_of_end, gsz(nch), 256, 0, st)(d_ends, nch, chain_of_end);
    CASL_K(k_ct_gather_chain, g, 256, 0, st)(term, ep, val, chain_of_end, d_pos, d_len, d_rot, d_cl,
                                             d_cc, xcr, ycr, ncr, rec);
  }
  CASL_K(k_walk_split, g, 256, 0, st)(rec, ncr, xw, yw, cidw);
  CASL_K(k_lev_of_contour, g, 256, 0, st)(startf, rlev, cidx, ncr, li, h->p.nlevm, clevt);
  RC_TRY(check_launch(h));

  tr.point("layout");
  RenodeIn cur{xw, yw, coff, clen, clevt, C, ncr, nullptr, cidw};
  if (econ) {
    // one periodic image of each contour, y folded (econgen.f90:238-252)
    int *flags = ar2.get<int>(C), *klen = ar2.get<int>(C), *kone = ar2.get<int>(C);
    int *koff = ar2.get<int>(C), *kidx = ar2.get<int>(C);
    int *cs2 = ar2.get<int>(C), *len2 = ar2.get<int>(C), *lev2 = ar2.get<int>(C);
    double *xw2 = ar2.get<double>(ncr), *yw2 = ar2.get<double>(ncr);
    int *cidw2 = ar2.get<int>(ncr);
    if (ar2.failed) return CASL_ENOMEM;
    CASL_CUDA_TRY(cudaMemsetAsync(flags, 0, (size_t)C * sizeof(int), st));
    CASL_K(k_ec_flags, g, 256, 0, st)(yw, cidw, ncr, c, flags);
    CASL_K(k_ec_keep, gsz(C), 256, 0, st)(flags, clen, C, klen, kone);
    exclusive_scan<int>(st, klen, koff, C, tmpi2, dtot + 4);
    exclusive_scan<int>(st, kone, kidx, C, tmpi2, dtot + 5);
    int kc[2] = {0, 0};
    CASL_CUDA_TRY(cudaMemcpyAsync(kc, dtot + 4, 2 * sizeof(int), cudaMemcpyDeviceToHost, st));
    CASL_CUDA_TRY(cudaStreamSynchronize(st));
    if (kc[1] == 0) return set_empty();
    const double yoff = c.hly + c.elly * (double)eg.nby;
    CASL_K(k_ec_compact, g, 256, 0, st)(xw, yw, cidw, ncr, coff, klen, koff, kidx, c, yoff, xw2,
                                        yw2, cidw2);
    CASL_K(k_ec_contours, gsz(C), 256, 0, st)(clen, clevt, C, klen, koff, kidx, cs2, len2, lev2);
    RC_TRY(check_launch(h));
    cur = RenodeIn{xw2, yw2, cs2, len2, lev2, kc[1], kc[0], nullptr, cidw2};
    tr.point("one image");
  }
  // --- 8. renode three times (congen.f90:295-310) -----------------------------
  long long capn = std::max<long long>(ncr * 2, h->npm);
  double *xa = ar2.get<double>(capn), *ya = ar2.get<double>(capn);
  double *xb = ar2.get<double>(capn), *yb = ar2.get<double>(capn);
  int *ocs[2], *olen[2], *olev[2];
  for (int q = 0; q < 2; q++) {
    ocs[q] = ar2.get<int>(C); olen[q] = ar2.get<int>(C); olev[q] = ar2.get<int>(C);
  }
  int *cnt = ar2.get<int>(4);
  if (ar2.failed) return CASL_ENOMEM;
  double *ox[3] = {xa, xb, xa}, *oy[3] = {ya, yb, ya};
  int hc[3] = {0, 0, 0};
  for (int pass = 0; pass < 3; pass++) {
    RenodeOut out{};
    out.xo = ox[pass]; out.yo = oy[pass];
    out.ocs = ocs[pass & 1]; out.olen = olen[pass & 1]; out.olev = olev[pass & 1];
    out.cap = capn;
    out.d_counts = cnt;
    size_t mark = ar2.off;
    RC_TRY(renode_batch(h, ar2, cur, out, RENODE_PLAIN));
    ar2.off = mark;
    CASL_CUDA_TRY(cudaMemcpyAsync(hc, cnt, 3 * sizeof(int), cudaMemcpyDeviceToHost, st));
    CASL_CUDA_TRY(cudaStreamSynchronize(st));
    if (hc[2]) return CASL_ECAPACITY;
    if (hc[0] == 0) return set_empty();
    cur = RenodeIn{out.xo, out.yo, out.ocs, out.olen, out.olev, hc[0], hc[1]};
    tr.point(pass == 0 ? "renode1" : (pass == 1 ? "renode2" : "renode3"));
  }
  int nq = hc[0], npt = hc[1];
  if (npt > h->npm || nq > h->nm) return CASL_ECAPACITY;
  CASL_CUDA_TRY(cudaMemcpyAsync(h->xq, cur.xw, (size_t)npt * sizeof(double), cudaMemcpyDeviceToDevice, st));
  CASL_CUDA_TRY(cudaMemcpyAsync(h->yq, cur.yw, (size_t)npt * sizeof(double), cudaMemcpyDeviceToDevice, st));
  CASL_K(k_out_contours, gsz(nq), 256, 0, st)(cur.cs, cur.len, cur.levt, nq, h->i1q, h->i2q, h->npq,
                                          h->indq);
  CASL_K(k_out_links, gsz(npt), 256, 0, st)(cur.cs, cur.len, nq, npt, h->nextq);
  CASL_K(k_set_counts2, 1, 1, 0, st)(h->scal, cnt);
  RC_TRY(check_launch(h));
  h->nq = nq;
  h->nptq = npt;
  h->contex = npt > 0;
  return CASL_OK;
}

}  // namespace casl

// ---------------------------------------------------------------------------
// genfg (post/genfg.f90:79-194): the PV on the ultra-fine grid as an image
// ---------------------------------------------------------------------------
namespace casl {

// out(iy, ix) = real(qa(iy1 + iy*stride, ix1 + ix*stride)), periodic, 0-based
// starts, out column-major (nyv, nxv)
__global__ void k_gf_gather(const double *__restrict__ qa, int nxu, int nyu, int ix1, int nxv,
                            int iy1, int nyv, int stride, float *__restrict__ out) {
  CASL_PDL_ENTRY();
  const long long m = (long long)nxv * nyv;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < m;
       t += (long long)gridDim.x * blockDim.x) {
    int iy = (int)(t % nyv), ix = (int)(t / nyv);
    long long sx = ((long long)ix1 + (long long)ix * stride) % nxu;
    long long sy = ((long long)iy1 + (long long)iy * stride) % nyu;
    out[t] = (float)qa[sx * nyu + sy];
  }
}

}  // namespace casl

using namespace casl;

extern "C" int casl_genfg(casl_handle *h, int ix1v, int nxv, int iy1v, int nyv, int stride,
                          float *out) {
  if (!h || !out) return CASL_EINVAL;
  if (h->M > 1) return CASL_EUNSUPPORTED;  // one simulation's image
  const Consts &c = h->c;
  const int nxu = c.nxu, nyu = c.nyu;
  if (ix1v < 1 || ix1v > nxu || iy1v < 1 || iy1v > nyu || nxv < 1 || nyv < 1 || stride < 1 ||
      (long long)(nxv - 1) * stride >= nxu || (long long)(nyv - 1) * stride >= nyu)
    return CASL_EINVAL;
  int rc = sync_counts(h);
  if (rc) return rc;
  cudaStream_t st = h->stream;
  const long long NU = (long long)nxu * nyu, m = (long long)nxv * nyv;
  size_t need = (size_t)NU * 12 + (size_t)nxu * 4 + (size_t)m * 4 + ((size_t)64 << 20);
  RC_TRY(ensure_scratch(h, need));
  Arena ar{(char *)h->sx, h->sx_bytes, 0};
  double *qa = ar.get<double>(NU);
  int *Lu = ar.get<int>(NU);
  int *ljx = ar.get<int>(nxu);
  unsigned long long *lsum = ar.get<unsigned long long>(4);
  double *part = ar.get<double>(2 * 4096);
  float *img = ar.get<float>(m);
  if (ar.failed) return CASL_ENOMEM;
  // con2ugrid (congen.f90:338-441), always called by genfg, then the
  // bilinear residual qr (genfg.f90:95-109)
  CASL_CUDA_TRY(cudaMemsetAsync(Lu, 0, (size_t)NU * sizeof(int), st));
  CASL_CUDA_TRY(cudaMemsetAsync(ljx, 0, (size_t)nxu * sizeof(int), st));
  CASL_CUDA_TRY(cudaMemsetAsync(lsum, 0, sizeof(unsigned long long), st));
  if (h->nptq > 0)
    CASL_K(k_u_scatter, gsz(h->nptq), 256, 0, st)(h->xq, h->yq, h->nextq, h->nptq, h->qjump, Lu,
                                              ljx, c, &h->scal->error);
  CASL_K(k_u_lbot, 1, 1024, 0, st)(ljx, Lu, nxu, nyu);
  CASL_K(k_u_colscan, (nxu * 32 + 255) / 256, 256, 0, st)(Lu, nxu, nyu, lsum);
  LevInfo lq{0, 0, h->qjump, 0.0, 1.0};
  CASL_K(k_u_field, 4096, 256, 0, st)(Lu, lsum, h->qr, h->qjump, 1, lq, qa, nullptr, part, c, 0.0);
  CASL_K(k_gf_gather, gsz(m), 256, 0, st)(qa, nxu, nyu, ix1v - 1, nxv, iy1v - 1, nyv, stride, img);
  RC_TRY(check_launch(h));
  CASL_CUDA_TRY(cudaMemcpyAsync(out, img, (size_t)m * sizeof(float), cudaMemcpyDeviceToHost, st));
  CASL_CUDA_TRY(cudaStreamSynchronize(st));
  return fetch_err(h);
}
