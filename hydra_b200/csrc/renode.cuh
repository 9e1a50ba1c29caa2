// Parallel node redistribution of many closed contours at once
// (renode, contours.f90:687-933).
//
// Input: contours stored contiguously in "walk order" (node k of contour c at
// cs[c] + k, the reference's xd(k+1)).  Every step of the reference's renode
// is a stencil over a node and its cyclic neighbours, so it runs one thread
// per node; the sequential "acc" walk that places new nodes becomes a
// segmented prefix sum of the node densities e(i) per contour, each old
// segment then emitting the new nodes whose cumulative density falls in it.
// Corners split a contour into pieces exactly as the reference's ncorn >= 2
// branch does.  Node counts (nint of the density sums) and the placement
// formula are the reference's; only the summation order of e(i) differs.
#pragma once

#include "common.cuh"
#include "scan.cuh"

namespace casl {

enum RenodeMode { RENODE_SURGERY = 0, RENODE_PLAIN = 1 };

struct RenodeIn {
  const double *xw, *yw;  // walk layout, N nodes
  const int *cs, *len;    // per contour
  const int *levt;        // per contour level index (copied to the output)
  int C;                  // contours (an upper bound when Cdev is given)
  long long N;            // nodes
  const int *Cdev;        // optional: the contour count in device memory
  const int *cid;         // optional: the contour of every walk node (else searched)
};

__device__ __forceinline__ int contours_in(const RenodeIn &in) { return in.Cdev ? *in.Cdev : in.C; }

struct RenodeOut {
  double *xo, *yo;        // output nodes (capacity cap)
  int *ocs, *olen, *olev; // output contours (capacity C)
  long long cap;
  int *d_counts;          // [0] contours kept, [1] nodes, [2] overflow flag
};

__device__ __forceinline__ int contour_of(const int *__restrict__ cs, int C, long long w) {
  int lo = 0, hi = C - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (cs[mid] <= w) lo = mid; else hi = mid - 1;
  }
  return lo;
}

struct RenodeScratch {
  int *cid;                  // contour of each walk node
  double *dx, *dy, *e, *A, *B, *Cc, *S;
  int *corner, *crank, *head;
  int *ccnt;                 // corners per contour
  double *ctot;              // density sum per contour
  int *npiece, *poff;        // pieces per contour, offsets
  int *pc, *pstart, *plen, *pn, *pout;  // per piece: contour, start w, length, count, out offset
  double *psum, *pfac;
  int *cnpr, *cout, *ckeep, *ckidx;     // per contour: kept npr, out offset, keep, kept index
  int *cornerpos;
  int *tmpi;
  SegPair *tmps;
  int *d_tot;
  long long maxpieces;
};

// Renodes every contour; issues no host synchronisation.  out.d_counts
// receives [kept contours, kept nodes, overflow flag]; on overflow (kept
// nodes > out.cap) nothing is written to the output arrays and the caller
// reports CASL_ECAPACITY when it reads the counts.
int renode_batch(casl_handle *h, Arena &ar, const RenodeIn &in, RenodeOut &out, int mode);

}  // namespace casl
