// Parallel renode of many contours (contours.f90:687-933); see renode.cuh.
#include <math.h>

#include "renode.cuh"

namespace casl {

__device__ __forceinline__ long long wnext(long long w, long long cs, long long L) {
  return w + 1 < cs + L ? w + 1 : cs;
}
__device__ __forceinline__ long long wprev(long long w, long long cs, long long L) {
  return w > cs ? w - 1 : cs + L - 1;
}

__global__ void k_rn_cid(RenodeIn in, long long N, int *__restrict__ cid) {
  CASL_PDL_ENTRY();
  const int C = contours_in(in);
  const int *cs = in.cs;
  for (long long w = blockIdx.x * (long long)blockDim.x + threadIdx.x; w < N;
       w += (long long)gridDim.x * blockDim.x)
    cid[w] = contour_of(cs, C, w);
}

// The node densities of renode (contours.f90:718-796) for node w: dx, dy,
// |d| to the next node; corners and curvature b; the cubic coefficients and
// spherical-curvature densities; node curvature as a weighted average; the
// fractional node count.  Only the results the placement reads (dx, dy, the
// final e, A, B, Cc, corner) go to memory.  rn_node recomputes every
// quantity node w needs from the coordinates of nodes w-2..w+3 (cyclic in
// the contour); k_rn_stencil computes each quantity once per node and passes
// it to the neighbouring lanes, with rn_node for the warps whose nodes come
// near a contour's end.  Both use the same expressions in the same order.
__device__ __forceinline__ void rn_node(const RenodeIn &in, const RenodeScratch &s, const Consts &c,
                                        long long w) {
  const double f12 = 0.5, f13 = 1.0 / 3.0, f16 = 1.0 / 6.0;
  const int k = s.cid[w];
  const long long cs = in.cs[k], L = in.len[k];
  long long j[6];
  j[2] = w;
  j[1] = wprev(w, cs, L);
  j[0] = wprev(j[1], cs, L);
  j[3] = wnext(w, cs, L);
  j[4] = wnext(j[3], cs, L);
  j[5] = wnext(j[4], cs, L);
  double X[6], Y[6];
#pragma unroll
  for (int m = 0; m < 6; m++) {
    X[m] = in.xw[j[m]];
    Y[m] = in.yw[j[m]];
  }
  // rn1 at nodes m = 0..4
  double dx[5], dy[5], v[5], e1[5];
#pragma unroll
  for (int m = 0; m < 5; m++) {
    double xx = X[m + 1] - X[m];
    dx[m] = xx - c.ellx * f_dint(xx * c.hlxi);
    double yy = Y[m + 1] - Y[m];
    dy[m] = yy - c.elly * f_dint(yy * c.hlyi);
    v[m] = dx[m] * dx[m] + dy[m] * dy[m];
    e1[m] = sqrt(v[m]);
  }
  // rn2 at nodes m = 1..4
  double b[5];
  int corner2 = 0;
#pragma unroll
  for (int m = 1; m < 5; m++) {
    double u = v[m - 1], a = -dx[m - 1], cc = -dy[m - 1];
    int corner = dx[m] * a + dy[m] * cc > 0.0;
    if (m == 2) corner2 = corner;
    if (corner) {
      b[m] = 0.0;
    } else {
      double t1 = a * v[m] - dx[m] * u, t2 = cc * v[m] - dy[m] * u;
      b[m] = (dx[m] * cc - a * dy[m]) / sqrt(t1 * t1 + t2 * t2 + c.small3);
    }
  }
  // rn3 at nodes m = 1..3 (the cubic coefficients only at m = 2)
  double u2[4], v2[4], A = 0.0, B = 0.0, Cc = 0.0;
#pragma unroll
  for (int m = 1; m < 4; m++) {
    double u = e1[m] * (b[m + 1] + b[m]);
    double cc = e1[m] * (b[m + 1] - b[m]);
    if (m == 2) {
      A = f16 * cc - f12 * u;
      B = f12 * (u - cc);
      Cc = f13 * cc;
    }
    double ww = 1.0 / (v[m] + c.dmsq);
    u2[m] = ww * sqrt(c.elf * v[m] + u * u);
    v2[m] = ww * e1[m];
  }
  // rn4 at nodes 2, 3 and rn5 at node 2
  const double d2 = (u2[1] + u2[2]) / (v2[1] + v2[2] + c.small);
  const double d3 = (u2[2] + u2[3]) / (v2[2] + v2[3] + c.small);
  const double uu = 0.5 * (d2 + d3);
  const double t = c.densf * sqrt(uu) + uu;
  s.dx[w] = dx[2];
  s.dy[w] = dy[2];
  s.e[w] = e1[2] * fmin(c.dmi, t);
  s.A[w] = A;
  s.B[w] = B;
  s.Cc[w] = Cc;
  s.corner[w] = corner2;
  s.head[w] = (w == cs);
  if (corner2) red_add_s32(&s.ccnt[k], 1);
}

// One warp covers nodes base-2 .. base+29 (lane L holds node base-2+L) and
// writes nodes base .. base+27 (lanes 2..29): the segment quantities (rn1)
// of lane L, its curvature (rn2), its cubic and density terms (rn3) and its
// rn4 average each take the lower neighbour's value from lane L-1 and the
// upper neighbour's from lane L+1.  Valid while every written node's
// stencil w-2..w+3 lies inside its contour without wrapping; otherwise the
// warp takes rn_node.
constexpr int RN_OUT = 28;
__global__ void __launch_bounds__(256, 4) k_rn_stencil(RenodeIn in, RenodeScratch s, Consts c) {
  CASL_PDL_ENTRY();
  const double f12 = 0.5, f13 = 1.0 / 3.0, f16 = 1.0 / 6.0;
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const long long N = in.N;
  const long long nwin = (N + RN_OUT - 1) / RN_OUT;
  const long long wstride = (long long)gridDim.x * (blockDim.x >> 5);
  for (long long wi = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); wi < nwin;
       wi += wstride) {
    const long long base = wi * RN_OUT;
    const long long o = base - 2 + lane;  // this lane's node
    const bool out = lane >= 2 && lane < 2 + RN_OUT && o < N;
    int k = 0;
    long long cs = 0, L = 0;
    bool lin = true;
    if (out) {
      k = s.cid[o];
      cs = in.cs[k];
      L = in.len[k];
      lin = o - 2 >= cs && o + 3 <= cs + L - 1;
    }
    if (!__all_sync(FULL, lin)) {
      if (out) rn_node(in, s, c, o);
      continue;
    }
    // coordinates of this lane's node and of the next one
    double X = 0.0, Y = 0.0, X1 = 0.0, Y1 = 0.0;
    if (o >= 0 && o < N) {
      X = in.xw[o];
      Y = in.yw[o];
    }
    if (lane == 31 && o + 1 < N) {
      X1 = in.xw[o + 1];
      Y1 = in.yw[o + 1];
    }
    double Xn = __shfl_down_sync(FULL, X, 1), Yn = __shfl_down_sync(FULL, Y, 1);
    if (lane == 31) {
      Xn = X1;
      Yn = Y1;
    }
    // rn1: the segment to the next node
    const double xx = Xn - X;
    const double dx = xx - c.ellx * f_dint(xx * c.hlxi);
    const double yy = Yn - Y;
    const double dy = yy - c.elly * f_dint(yy * c.hlyi);
    const double v = dx * dx + dy * dy;
    const double e1 = sqrt(v);
    // rn2 at this node, from the previous segment
    const double up = __shfl_up_sync(FULL, v, 1);
    const double a = -__shfl_up_sync(FULL, dx, 1), ccp = -__shfl_up_sync(FULL, dy, 1);
    const int corner = dx * a + dy * ccp > 0.0;
    double b;
    if (corner) {
      b = 0.0;
    } else {
      const double t1 = a * v - dx * up, t2 = ccp * v - dy * up;
      b = (dx * ccp - a * dy) / sqrt(t1 * t1 + t2 * t2 + c.small3);
    }
    // rn3 at this node, with the next node's curvature
    const double bn = __shfl_down_sync(FULL, b, 1);
    const double u = e1 * (bn + b);
    const double cc = e1 * (bn - b);
    const double A = f16 * cc - f12 * u;
    const double B = f12 * (u - cc);
    const double Cc = f13 * cc;
    const double ww = 1.0 / (v + c.dmsq);
    const double u2 = ww * sqrt(c.elf * v + u * u);
    const double v2 = ww * e1;
    // rn4 at this node (with the previous node's rn3) and at the next one
    const double u2p = __shfl_up_sync(FULL, u2, 1), v2p = __shfl_up_sync(FULL, v2, 1);
    const double d = (u2p + u2) / (v2p + v2 + c.small);
    const double dn = __shfl_down_sync(FULL, d, 1);
    if (out) {
      // rn5
      const double uu = 0.5 * (d + dn);
      const double t = c.densf * sqrt(uu) + uu;
      s.dx[o] = dx;
      s.dy[o] = dy;
      s.e[o] = e1 * fmin(c.dmi, t);
      s.A[o] = A;
      s.B[o] = B;
      s.Cc[o] = Cc;
      s.corner[o] = corner;
      s.head[o] = (o == cs);
      if (corner) red_add_s32(&s.ccnt[k], 1);
    }
  }
}

__global__ void k_rn_cornerpos(const int *__restrict__ corner, const int *__restrict__ crank,
                               int *__restrict__ pos, long long N) {
  CASL_PDL_ENTRY();
  for (long long w = blockIdx.x * (long long)blockDim.x + threadIdx.x; w < N;
       w += (long long)gridDim.x * blockDim.x)
    if (corner[w]) pos[crank[w]] = (int)w;
}

// Sum of e over `m` nodes of contour [cs, cs+L) starting at walk index st.
__device__ __forceinline__ double sumrange(const double *__restrict__ S, long long cs,
                                           long long L, long long st, long long m) {
  long long a = st - cs, b = a + m;
  auto pre = [&](long long k) -> double { return k == 0 ? 0.0 : S[cs + k - 1]; };
  if (b <= L) return pre(b) - pre(a);
  return (pre(L) - pre(a)) + pre(b - L);
}

__device__ __forceinline__ int nint_d(double x) { return (int)llround(x); }

// The reference adds a contour's (or a corner piece's) densities one after
// the other from its first node (contours.f90:799-806, 843-853) and rounds
// the total to the node count.  The prefix sums here group the additions
// otherwise; where the total lies within 1e-6 of a half-integer, so that
// the grouping could move it across the rounding point, it is recomputed in
// the reference's order: m densities from node st, wrapping within
// [cs, cs+L).
__device__ __forceinline__ bool near_half(double x) {
  const double f = x - floor(x);
  return fabs(f - 0.5) < 1e-6;
}
__device__ double seq_sum(const double *__restrict__ e, long long cs, long long L, long long st,
                          long long m) {
  double t = 0.0;
  long long i = st - cs;
  for (long long j = 0; j < m; j++) {
    t = t + e[cs + i];
    if (++i == L) i = 0;
  }
  return t;
}

// Per contour: node count, pieces (contours.f90:799-809, 813-930), and
// where its pieces are stored (block by block from a running total in
// d_tot[1]; piece storage order is free, the output order comes from the
// contour scan).
__global__ void k_rn_count(RenodeIn in, RenodeScratch s, Consts c, int mode) {
  CASL_PDL_ENTRY();
  __shared__ int btot, bbase;
  const int Ce = contours_in(in);
  for (int base = blockIdx.x * blockDim.x; base < Ce; base += gridDim.x * blockDim.x) {
    const int k = base + threadIdx.x;
    int np = 0;
    if (k < Ce) {
      long long cs = in.cs[k], L = in.len[k];
      double total = s.S[cs + L - 1];
      if (near_half(total)) total = seq_sum(s.e, cs, L, cs, L);
      s.ctot[k] = total;
      if (!(mode == RENODE_SURGERY && L <= 3)) {
        int npr0 = nint_d(total) + 1;
        if (npr0 >= 3) np = s.ccnt[k] > 1 ? s.ccnt[k] : 1;
      }
      s.npiece[k] = np;
    }
    const int ex = block_excl_scan_any<int>(np, &btot);
    if (threadIdx.x == 0) bbase = atomicAdd(&s.d_tot[1], btot);
    __syncthreads();
    if (k < Ce) s.poff[k] = bbase + ex;
    __syncthreads();
  }
}

__global__ void k_rn_fill(RenodeIn in, RenodeScratch s, Consts c, int mode) {
  CASL_PDL_ENTRY();
  const int Ce = contours_in(in);
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < Ce; k += gridDim.x * blockDim.x) {
    long long cs = in.cs[k], L = in.len[k];
    int np = s.npiece[k];
    int npr = 0;
    double total = s.ctot[k];
    int nc = s.ccnt[k];
    int cfirst = s.crank[cs];
    for (int q = 0; q < np; q++) {
      int p = s.poff[k] + q;
      long long st, pl;
      double sum;
      int n;
      if (nc <= 1) {
        st = nc == 0 ? cs : s.cornerpos[cfirst];
        pl = L;
        sum = total;
        n = nint_d(total) + 1;
      } else {
        st = s.cornerpos[cfirst + q];
        long long en = s.cornerpos[cfirst + (q + 1) % nc];
        pl = en - st;  // both corners lie in [cs, cs+L)
        if (pl < 0) pl += L;
        sum = sumrange(s.S, cs, L, st, pl);
        if (near_half(sum)) sum = seq_sum(s.e, cs, L, st, pl);
        n = sum > c.small ? nint_d(sum) + 1 : 0;
      }
      s.pc[p] = k;
      s.pstart[p] = (int)st;
      s.plen[p] = (int)pl;
      s.psum[p] = sum;
      s.pn[p] = n;
      s.pfac[p] = n > 0 ? (double)n / sum : 0.0;
      npr += n;
    }
    int keep = mode == RENODE_SURGERY ? npr > 3 : npr > 0;
    s.ckeep[k] = keep;
    s.cnpr[k] = keep ? npr : 0;
  }
}

__global__ void k_rn_pout(RenodeIn in, RenodeScratch s, RenodeOut out) {
  CASL_PDL_ENTRY();
  if (out.d_counts[2]) return;  // overflow: the caller reports it
  const int Ce = contours_in(in);
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < Ce; k += gridDim.x * blockDim.x) {
    if (!s.ckeep[k]) continue;
    int base = s.cout[k];
    for (int q = 0; q < s.npiece[k]; q++) {
      int p = s.poff[k] + q;
      s.pout[p] = base;
      base += s.pn[p];
    }
    int j = s.ckidx[k];
    out.ocs[j] = s.cout[k];
    out.olen[j] = s.cnpr[k];
    out.olev[j] = in.levt ? in.levt[k] : 0;
  }
}

__global__ void k_rn_place(RenodeIn in, RenodeScratch s, RenodeOut out, Consts c) {
  CASL_PDL_ENTRY();
  if (out.d_counts[2]) return;  // overflow: the caller reports it
  for (long long w = blockIdx.x * (long long)blockDim.x + threadIdx.x; w < in.N;
       w += (long long)gridDim.x * blockDim.x) {
    int k = s.cid[w];
    if (!s.ckeep[k]) continue;
    long long cs = in.cs[k], L = in.len[k];
    int nc = s.ccnt[k];
    int q = 0;
    if (nc >= 2) {
      int inc = s.crank[w] - s.crank[cs] + s.corner[w];
      q = inc - 1;
      if (q < 0) q = nc - 1;
    }
    int p = s.poff[k] + q;
    int n = s.pn[p];
    if (n == 0) continue;
    long long st = s.pstart[p];
    // w and the piece start both lie in the contour [cs, cs+L)
    long long rel = w - st;
    if (rel < 0) rel += L;
    if (rel >= s.plen[p]) continue;
    long long o = s.pout[p];
    if (rel == 0) {
      out.xo[o] = in.xw[w];
      out.yo[o] = in.yw[w];
    }
    double fac = s.pfac[p];
    double Ep = fac * sumrange(s.S, cs, L, st, rel);
    double Ec = fac * sumrange(s.S, cs, L, st, rel + 1);
    long long t0 = (long long)floor(Ep) + 1;
    long long t1 = (long long)floor(Ec);
    if (t1 > n - 1) t1 = n - 1;
    if (t0 < 1) t0 = 1;
    if (t1 < t0) continue;
    double ew = fac * s.e[w];
    double xd = in.xw[w], yd = in.yw[w], dx = s.dx[w], dy = s.dy[w];
    double A = s.A[w], B = s.B[w], Cc = s.Cc[w];
    for (long long t = t0; t <= t1; t++) {
      double acc = Ec - (double)t;
      double pp = 1.0 - acc / ew;
      // Targets are assigned by prefix sums, whose grouping rounds: a
      // segment of density zero or at the rounding level (the zero-length
      // segments that surgery leaves where it joins two nodes) can receive
      // a target that the reference's running sum gives its neighbour, and
      // 1 - acc/ew is then far outside [0, 1] or 0/0.  Such a target is
      // placed by the prefix values that assigned it (Ep < t <= Ec, so the
      // fraction lies in (0, 1]): the segment's start, within rounding of
      // where the reference puts it.
      if (!(pp >= -1e-9 && pp <= 1.0 + 1e-9)) pp = ((double)t - Ep) / (Ec - Ep);
      double eta = pp * (A + pp * (B + pp * Cc));
      double xx = xd + pp * dx - eta * dy;
      double yy = yd + pp * dy + eta * dx;
      out.xo[o + t] = wrapp(xx, c.ellx, c.hlxi, c.oms);
      out.yo[o + t] = wrapp(yy, c.elly, c.hlyi, c.oms);
    }
  }
}

// The kept contours' node counts and keep flags scanned (both over the
// contours the device holds), then the output counts: one block.
__global__ void __launch_bounds__(SCAN_BLOCK) k_rn_scan2_finish(RenodeIn in, RenodeScratch s,
                                                                RenodeOut out) {
  CASL_PDL_ENTRY();
  __shared__ unsigned long long tot;
  const long long n = contours_in(in);
  // each thread takes a run of consecutive contours; both counts go through
  // one scan, the node counts in the high word and the keep flags in the low
  // word (each total stays below 2^31)
  auto pack = [&](long long k) -> unsigned long long {
    return ((unsigned long long)(unsigned)s.cnpr[k] << 32) | (unsigned)s.ckeep[k];
  };
  const long long per = (n + SCAN_BLOCK - 1) / SCAN_BLOCK;
  const long long k0 = min(n, (long long)threadIdx.x * per), k1 = min(n, k0 + per);
  unsigned long long sum = 0;
  for (long long k = k0; k < k1; k++) sum += pack(k);
  unsigned long long ex = block_excl_scan<unsigned long long>(sum, &tot);
  for (long long k = k0; k < k1; k++) {
    s.cout[k] = (int)(ex >> 32);
    s.ckidx[k] = (int)(ex & 0xffffffffu);
    ex += pack(k);
  }
  if (threadIdx.x == 0) {
    const long long nodes = (long long)(tot >> 32);
    out.d_counts[0] = (int)(tot & 0xffffffffu);
    out.d_counts[1] = (int)nodes;
    out.d_counts[2] = nodes > out.cap;
  }
}

static inline int gsz(long long work) {
  long long g = (work + 255) / 256;
  if (g < 1) g = 1;
  if (g > 148 * 16) g = 148 * 16;
  return (int)g;
}

int renode_batch(casl_handle *h, Arena &ar, const RenodeIn &in, RenodeOut &out, int mode) {
  cudaStream_t st = h->stream;
  const Consts &c = h->c;
  long long N = in.N;
  int C = in.C;  // capacity when in.Cdev is set
  if (C == 0 || N == 0) {
    cudaMemsetAsync(out.d_counts, 0, 3 * sizeof(int), st);
    return CASL_OK;
  }
  RenodeScratch s{};
  s.cid = in.cid ? const_cast<int *>(in.cid) : ar.get<int>(N);
  s.dx = ar.get<double>(N); s.dy = ar.get<double>(N);
  s.e = ar.get<double>(N); s.A = ar.get<double>(N);
  s.B = ar.get<double>(N); s.Cc = ar.get<double>(N); s.S = ar.get<double>(N);
  s.corner = ar.get<int>(N); s.crank = ar.get<int>(N); s.head = ar.get<int>(N);
  s.cornerpos = ar.get<int>(N + 1);
  s.ccnt = ar.get<int>(C); s.ctot = ar.get<double>(C);
  s.npiece = ar.get<int>(C); s.poff = ar.get<int>(C);
  s.cnpr = ar.get<int>(C); s.cout = ar.get<int>(C); s.ckeep = ar.get<int>(C);
  s.ckidx = ar.get<int>(C);
  long long tmpn = scan_tmp_elems(N > C ? N : C) + 4;
  s.tmpi = ar.get<int>(tmpn);
  s.tmps = ar.get<SegPair>(tmpn);
  s.d_tot = ar.get<int>(8);
  // pieces: one per corner of a contour with >= 2 corners, else one per
  // contour, so at most N + C
  long long P = N + C;
  s.pc = ar.get<int>(P); s.pstart = ar.get<int>(P); s.plen = ar.get<int>(P);
  s.pn = ar.get<int>(P); s.pout = ar.get<int>(P);
  s.psum = ar.get<double>(P); s.pfac = ar.get<double>(P);
  if (ar.failed) return CASL_ENOMEM;
  {
    const FillJob z[2] = {{s.ccnt, C, 0u}, {s.d_tot + 1, 1, 0u}};
    if (int rc = fill_words(st, z, 2)) return rc;
  }
  int g = gsz(N);
  if (!in.cid) CASL_K(k_rn_cid, g, 256, 0, st)(in, N, s.cid);
  CASL_K(k_rn_stencil, g, 256, 0, st)(in, s, c);
  segmented_scan(st, s.e, s.head, s.S, N, s.tmps);
  exclusive_scan<int>(st, s.corner, s.crank, N, s.tmpi, s.d_tot + 0);
  CASL_K(k_rn_cornerpos, g, 256, 0, st)(s.corner, s.crank, s.cornerpos, N);
  // per-contour passes: C may be a capacity (surgery: the count is on the
  // device), so the grids are sized for the usual counts and loop
  int gc = gsz(C < (1 << 16) ? C : (1 << 16));
  CASL_K(k_rn_count, gc, 256, 0, st)(in, s, c, mode);
  CASL_K(k_rn_fill, gc, 256, 0, st)(in, s, c, mode);
  CASL_K(k_rn_scan2_finish, 1, SCAN_BLOCK, 0, st)(in, s, out);
  CASL_K(k_rn_pout, gc, 256, 0, st)(in, s, out);
  CASL_K(k_rn_place, g, 256, 0, st)(in, s, out, c);
  return check_launch(h);
}

}  // namespace casl
