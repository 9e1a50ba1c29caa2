// Batched real FFTs in the stafft "Hermitian" layout, one axis at a time.
//
// The transform restated (lib/stafft/stafft.f90:55-58,187-406):
//   forward:  X[k]   = Re F(k) / sqrt(n)   k = 0..n/2
//             X[n-k] = Im F(k) / sqrt(n)   k = 1..n/2-1,  F(k) = sum_j x_j e^{-2 pi i jk/n}
//   reverse:  the exact inverse.
// A 2-D ptospc/spctop (sta2dfft.f90:103-165) is two launches of this kernel,
// one per axis, with the transpose folded into the store/load addressing.
//
// B200 design: one CTA transforms V vectors of one field on chip.  The real
// length-n transform runs as a complex length-n/2 Stockham FFT (radix 8,
// then 4 or 2) bracketed by the even/odd untangling step.  Global traffic is
// exactly one read and one write of every element per axis; the load and
// store are functors so that pointwise spectral work (Green function,
// derivatives, filters, products) fuses into the transform instead of
// costing extra HBM passes.  LVF / SVF: whether consecutive vectors (true)
// or consecutive elements (false) are adjacent in global memory for the load
// / the store, which sets the thread mapping for coalescing.
#pragma once

#include <type_traits>

#include "common.cuh"
#include "hydra_casl.h"
#include "tc.cuh"

namespace casl {

__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
// Complex product with fused multiply-adds (transform outputs are compared
// to the oracle within a tolerance, not bit for bit).
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(__fma_rn(a.x, b.x, -(a.y * b.y)), __fma_rn(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
// multiply by -i (FWD) or +i (inverse)
template <bool FWD>
__device__ __forceinline__ double2 mul_mi(double2 a) {
  return FWD ? make_double2(a.y, -a.x) : make_double2(-a.y, a.x);
}

template <bool FWD>
__device__ __forceinline__ void dft2(double2 *v) {
  double2 a = v[0], b = v[1];
  v[0] = cadd(a, b);
  v[1] = csub(a, b);
}

template <bool FWD>
__device__ __forceinline__ void dft4(double2 &v0, double2 &v1, double2 &v2, double2 &v3) {
  double2 a = cadd(v0, v2), b = csub(v0, v2), c = cadd(v1, v3), d = mul_mi<FWD>(csub(v1, v3));
  v0 = cadd(a, c);
  v2 = csub(a, c);
  v1 = cadd(b, d);
  v3 = csub(b, d);
}

template <bool FWD>
__device__ __forceinline__ void dft8(double2 *v) {
  // even / odd radix-4 halves, then combine with w8^k
  double2 e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
  double2 o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
  dft4<FWD>(e0, e1, e2, e3);
  dft4<FWD>(o0, o1, o2, o3);
  const double r = 0.70710678118654752440084436210484903928483593768847;
  // w8^1 = (1 -+ i) r ; w8^2 = -+i ; w8^3 = (-1 -+ i) r
  double2 t1 = FWD ? make_double2(r * (o1.x + o1.y), r * (o1.y - o1.x))
                   : make_double2(r * (o1.x - o1.y), r * (o1.y + o1.x));
  double2 t2 = mul_mi<FWD>(o2);
  double2 t3 = FWD ? make_double2(r * (o3.y - o3.x), -r * (o3.x + o3.y))
                   : make_double2(-r * (o3.x + o3.y), r * (o3.x - o3.y));
  v[0] = cadd(e0, o0);
  v[4] = csub(e0, o0);
  v[1] = cadd(e1, t1);
  v[5] = csub(e1, t1);
  v[2] = cadd(e2, t2);
  v[6] = csub(e2, t2);
  v[3] = cadd(e3, t3);
  v[7] = csub(e3, t3);
}

// A load functor may also provide pair(b, v, j) -> elements (j, j+1) for
// even j, and a store functor pair(b, v, k, x) for (k, k+1): one 16-byte
// access instead of two 8-byte ones where the elements are adjacent.
template <class T, class = void>
struct has_pair : std::false_type {};
template <class T>
struct has_pair<T, std::void_t<decltype(&T::pair)>> : std::true_type {};

// a[b] for a functor's small per-batch array without indexing it at run
// time: an indexed kernel-parameter array is copied to local memory and
// every use costs a local load in front of the global one; the unrolled
// select keeps the entries in the parameter bank.
template <class T, int N>
__device__ __forceinline__ T pick(const T (&a)[N], int b) {
  T r = a[0];
#pragma unroll
  for (int i = 1; i < N; i++)
    if (b == i) r = a[i];
  return r;
}

// Plain strided load / store functors: element (b, v, j) at p[b*bs + v*vs + j*es].
struct LoadStrided {
  __host__ double bytes() const { return 8.0; }
  const double *p;
  long long bs, vs, es;
  __device__ __forceinline__ double operator()(int b, int v, int j) const {
    return p[b * bs + (long long)v * vs + (long long)j * es];
  }
  __device__ __forceinline__ double2 pair(int b, int v, int j) const {
    const long long o = b * bs + (long long)v * vs + (long long)j * es;
    if (es == 1) return *reinterpret_cast<const double2 *>(p + o);
    return make_double2(p[o], p[o + es]);
  }
};
// A contiguous row per vector, element (b, v, j) at p[b*bs + v*vs + j]: the
// plain load of a pass whose load side is element-contiguous, staged in
// shared memory by one bulk copy per vector (see has_rows below).
struct LoadRow {
  __host__ double bytes() const { return 8.0; }
  const double *p;
  long long bs, vs;
  int n;
  int *err = nullptr;
  static constexpr int NROWS = 1;
  __device__ __forceinline__ double operator()(int b, int v, int j) const {
    return p[b * bs + (long long)v * vs + j];
  }
  __device__ __forceinline__ uint32_t stage_bytes(int, int) const { return (uint32_t)n * 8u; }
  __device__ __forceinline__ void stage(int b, int v, double *dst, uint64_t *bar) const {
    tc::bulk_g2s(dst, p + b * bs + (long long)v * vs, (uint32_t)n * 8u, bar);
  }
  __device__ __forceinline__ void fail() const {
    if (err) atomicExch(err, CASL_ETIMEOUT);
  }
  __device__ __forceinline__ double staged(int, int, int j, const double *R) const { return R[j]; }
};
struct StoreStrided {
  __host__ double bytes() const { return 8.0; }
  double *p;
  long long bs, vs, es;
  __device__ __forceinline__ void operator()(int b, int v, int k, double x) const {
    p[b * bs + (long long)v * vs + (long long)k * es] = x;
  }
  __device__ __forceinline__ void pair(int b, int v, int k, double2 x) const {
    const long long o = b * bs + (long long)v * vs + (long long)k * es;
    if (es == 1) {
      *reinterpret_cast<double2 *>(p + o) = x;
    } else {
      p[o] = x.x;
      p[o + es] = x.y;
    }
  }
};

// ---------------------------------------------------------------------------
// Register-resident transform.  Each vector of complex length H = 2^LOGH is
// handled by H/8 threads holding 8 complex values each; a radix-8 (or the
// final radix-4/2) butterfly runs in registers and only the exchange between
// passes goes through one shared slot per vector, so shared traffic is a
// single write + read per pass instead of a ping-pong of whole buffers.
// Where global memory is element-contiguous (LVF / SVF false) the loads and
// stores go straight between registers and HBM, coalesced across the
// vector's threads; vector-fastest layouts are staged through shared memory
// with lanes running over vectors.
//
// Register convention: before and after every pass thread t holds
// x[m] = Z[t + m*TPV], m = 0..7 (TPV = H/8).  A radix-R pass applies 8/R
// butterflies j = t + m*TPV on x[m + r*(8/R)], r = 0..R-1, which are exactly
// the Stockham inputs j + r*H/R; for the last pass (Ns*R = H) the outputs
// j + r*Ns land back in the same slots, so only earlier passes scatter.
// Padded position of complex element i within a slot: one spare element per
// eight keeps the stride-8 scatter of the first pass conflict-free.
__device__ __forceinline__ int cpad(int i) { return i + (i >> 3); }
__device__ __forceinline__ int dpos(int j) { return 2 * cpad(j >> 1) + (j & 1); }

// VF: a side of the pass is vector-fastest and is staged through shared
// memory with lanes over vectors, which wants several vectors per CTA (V*8
// contiguous bytes per row); contiguous-only passes take small CTAs so that
// one transform spreads evenly over all SMs.
template <int LOGH, bool VF>
struct RfftShape {
  static constexpr int H = 1 << LOGH;
  static constexpr int N = 2 * H;
  static constexpr int TPV = H / 8;
  static constexpr int VS = H + H / 8 + 1;  // complex stride between slots
  static constexpr int VW = VF ? 256 / TPV : 64 / TPV;
  static constexpr int V = VW < 1 ? 1 : (VW < N ? VW : N);  // vectors per CTA
  static constexpr int NT = V * TPV;        // threads per CTA
  // CTAs per SM to fit: 1024 threads (<= 64 registers; a little faster in
  // the step than 768 threads at 80 registers)
  static constexpr int MINB = 1024 / NT > 0 ? 1024 / NT : 1;
  static constexpr int P8 = LOGH / 3;       // radix-8 passes
  static constexpr int REM = LOGH % 3;      // final radix-4 (2) or radix-2 (1) pass
  // forward transforms with a vector-fastest store stage their output in a
  // second region, so the untangle can emit while other threads still read Z
  static constexpr size_t smem(bool fwd_svf) {
    return (size_t)(fwd_svf ? 2 : 1) * V * VS * sizeof(double2);
  }
};

template <int R, bool FWD, int TPV>
__device__ __forceinline__ void rf_butterflies(double2 (&x)[8], int t, int Ns,
                                               const double2 *__restrict__ tw, int n) {
  constexpr int NB = 8 / R;
#pragma unroll
  for (int m = 0; m < NB; m++) {
    double2 y[R];
#pragma unroll
    for (int r = 0; r < R; r++) y[r] = x[m + r * NB];
    const int j = t + m * TPV;
    const int k = j & (Ns - 1);
    if (k) {
      // powers w^r of the butterfly's twiddle w (one table load): products
      // at most three deep, so each is within a few ulps
      const int ts = n / (Ns * R);
      double2 wr[8];
      wr[1] = __ldg(&tw[k * ts]);
      if (R >= 4) wr[2] = cmul(wr[1], wr[1]);
      if (R == 8) wr[4] = cmul(wr[2], wr[2]);
      if (R >= 4) wr[3] = cmul(wr[1], wr[2]);
      if (R == 8) {
        wr[5] = cmul(wr[1], wr[4]);
        wr[6] = cmul(wr[2], wr[4]);
        wr[7] = cmul(wr[3], wr[4]);
      }
#pragma unroll
      for (int r = 1; r < R; r++) y[r] = cmul(y[r], FWD ? wr[r] : cconj(wr[r]));
    }
    if (R == 8) dft8<FWD>(y);
    if (R == 4) dft4<FWD>(y[0], y[1], y[2], y[3]);
    if (R == 2) dft2<FWD>(y);
#pragma unroll
    for (int r = 0; r < R; r++) x[m + r * NB] = y[r];
  }
}

// All passes of the complex FFT; x holds Z[t + m*TPV] on entry and on exit.
// S is this vector's slot; the caller has synchronised after its last read
// of shared memory.
template <int LOGH, bool FWD>
__device__ __forceinline__ void rf_complex(double2 (&x)[8], double2 *S, int t,
                                           const double2 *__restrict__ tw, int n) {
  using Sh = RfftShape<LOGH, false>;  // only H, TPV and the pass plan are used
  int Ns = 1;
#pragma unroll
  for (int p = 0; p < Sh::P8; p++) {
    rf_butterflies<8, FWD, Sh::TPV>(x, t, Ns, tw, n);
    if (p < Sh::P8 - 1 || Sh::REM != 0) {
      const int base = (t / Ns) * Ns * 8 + (t & (Ns - 1));
#pragma unroll
      for (int r = 0; r < 8; r++) S[cpad(base + r * Ns)] = x[r];
      __syncthreads();
#pragma unroll
      for (int m = 0; m < 8; m++) x[m] = S[cpad(t + m * Sh::TPV)];
      __syncthreads();
    }
    Ns *= 8;
  }
  if (Sh::REM == 2) rf_butterflies<4, FWD, Sh::TPV>(x, t, Ns, tw, n);
  if (Sh::REM == 1) rf_butterflies<2, FWD, Sh::TPV>(x, t, Ns, tw, n);
}

// A load functor with a static member NROWS (1 or 2) stages its input rows
// in shared memory by bulk copies instead of loading elements one by one: in
// a pass whose load side is element-contiguous, vector v of batch entry b
// reads NROWS rows of n doubles, which stage(b, v, dst, bar) copies to dst
// (NROWS * n doubles) against the barrier, returning the bytes it copies;
// staged(b, v, j, rows) then gives element j from them.  The copies put a
// whole vector's input in flight at once without holding registers, where
// element loads left the pass bound by load latency.  A copy that does not
// arrive in about a second is reported through fail().
template <class T, class = void>
struct has_rows : std::false_type {};
template <class T>
struct has_rows<T, std::void_t<decltype(T::NROWS)>> : std::true_type {};
template <class LD, bool LVF>
constexpr int staged_rows() {
  if constexpr (has_rows<LD>::value && !LVF) return LD::NROWS;
  else return 0;
}

// A load or store functor may ask for fewer CTAs per SM (more registers)
// through a static member `wide`: the derivative load keeps 80 registers,
// where 64 would spill.
template <class T, class = void>
struct wants_wide : std::false_type {};
template <class T>
struct wants_wide<T, std::void_t<decltype(T::wide)>> : std::bool_constant<T::wide> {};
template <int LOGH, bool VF, class LD, class ST>
constexpr int rfft_minb() {
  using Sh = RfftShape<LOGH, VF>;
  return (wants_wide<LD>::value || wants_wide<ST>::value) ? (768 / Sh::NT > 0 ? 768 / Sh::NT : 1)
                                                          : Sh::MINB;
}

// Shared memory of a pass: the exchange (and forward staging) regions, or
// the staged input rows over them where larger, then the staging barrier.
template <int LOGH, bool FWD, bool LVF, bool SVF, int NR>
constexpr size_t rfft_bar_offset() {
  using Sh = RfftShape<LOGH, LVF || SVF>;
  const size_t ex = Sh::smem(FWD && SVF);
  const size_t rows = (size_t)Sh::V * NR * Sh::N * sizeof(double);
  return ((ex > rows ? ex : rows) + 15) / 16 * 16;
}
template <int LOGH, bool FWD, bool LVF, bool SVF, int NR>
constexpr size_t rfft_smem() {
  using Sh = RfftShape<LOGH, LVF || SVF>;
  return NR ? rfft_bar_offset<LOGH, FWD, LVF, SVF, NR>() + 16 : Sh::smem(FWD && SVF);
}

template <int LOGH, bool FWD, bool LVF, bool SVF, class LD, class ST>
__global__ void __launch_bounds__(RfftShape<LOGH, LVF || SVF>::NT,
                                  (rfft_minb<LOGH, LVF || SVF, LD, ST>()))
    k_rfft_r(LD ld, ST st, const double2 *__restrict__ tw) {
  CASL_PDL_ENTRY();
  using Sh = RfftShape<LOGH, LVF || SVF>;
  constexpr int H = Sh::H, N = Sh::N, TPV = Sh::TPV, V = Sh::V, NT = Sh::NT, VS = Sh::VS;
  extern __shared__ double2 smem[];
  double *Sd = reinterpret_cast<double *>(smem);
  const int vl = threadIdx.x / TPV, t = threadIdx.x - vl * TPV;
  const int v0 = blockIdx.x * V, vg = v0 + vl;
  const int b = blockIdx.y;
  double2 *S = smem + vl * VS;
  double *SdV = Sd + 2 * vl * VS;
  double2 x[8];

  // Bulk-staged contiguous input: this CTA's V vectors' rows at the start
  // of shared memory, over the exchange (and forward staging) regions, which
  // are first written after every thread has read its inputs; the barrier
  // after both.
  constexpr int NR = staged_rows<LD, LVF>();
  [[maybe_unused]] const double *Rw = nullptr;
  if constexpr (NR > 0) {
    double *R0 = Sd;
    uint64_t *bar = reinterpret_cast<uint64_t *>(
        reinterpret_cast<unsigned char *>(smem) + rfft_bar_offset<LOGH, FWD, LVF, SVF, NR>());
    Rw = R0 + vl * NR * N;
    if (threadIdx.x == 0) {
      tc::mbar_init(bar, 1);
      tc::mbar_fence_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      uint32_t bytes = 0;
#pragma unroll 1
      for (int q = 0; q < V; q++) bytes += ld.stage_bytes(b, v0 + q);
      tc::mbar_expect_tx(bar, bytes);
#pragma unroll 1
      for (int q = 0; q < V; q++) ld.stage(b, v0 + q, R0 + q * NR * N, bar);
    }
    if (!tc::mbar_wait(bar, 0) && threadIdx.x == 0) ld.fail();
  }

  // Vector-fastest input: stage V vectors, lanes over vectors (16 values per
  // thread, loaded 8 at a time).
  if (LVF) {
    constexpr int Q = (V * N) / NT;
#pragma unroll
    for (int q0 = 0; q0 < Q; q0 += 8) {
      double r[8];
#pragma unroll
      for (int q = 0; q < 8; q++) {
        int idx = threadIdx.x + (q0 + q) * NT;
        r[q] = ld(b, v0 + (idx % V), idx / V);
      }
#pragma unroll
      for (int q = 0; q < 8; q++) {
        int idx = threadIdx.x + (q0 + q) * NT;
        Sd[2 * (idx % V) * VS + dpos(idx / V)] = r[q];
      }
    }
    __syncthreads();
  }

  if (FWD) {
    if (LVF) {
#pragma unroll
      for (int m = 0; m < 8; m++) x[m] = S[cpad(t + m * TPV)];
      __syncthreads();
    } else {
#pragma unroll
      for (int m = 0; m < 8; m++) {
        int e = t + m * TPV;
        if constexpr (NR > 0)
          x[m] = make_double2(ld.staged(b, vg, 2 * e, Rw), ld.staged(b, vg, 2 * e + 1, Rw));
        else if constexpr (has_pair<LD>::value)
          x[m] = ld.pair(b, vg, 2 * e);
        else
          x[m] = make_double2(ld(b, vg, 2 * e), ld(b, vg, 2 * e + 1));
      }
      if constexpr (NR > 0) __syncthreads();  // rows read before the slots overwrite them
    }
    rf_complex<LOGH, true>(x, S, t, tw, N);
    // untangle: pairs (k, H-k) live in threads t and TPV-t, so exchange once
#pragma unroll
    for (int m = 0; m < 8; m++) S[cpad(t + m * TPV)] = x[m];
    __syncthreads();
    const double s = 1.0 / sqrt((double)N);
    double *Out = Sd + 2 * V * VS + 2 * vl * VS;  // forward + SVF staging region
    auto emit = [&](int k, double val) {
      if (SVF) Out[dpos(k)] = val; else st(b, vg, k, val);
    };
    // tw[H-k] = -conj(tw[k]) (tw[H] = -1), so a pair needs one table load
    auto pair_out = [&](int kk, double2 w) {
      double2 zk = S[cpad(kk)], zc = cconj(S[cpad(H - kk)]);
      double2 e = make_double2(0.5 * (zk.x + zc.x), 0.5 * (zk.y + zc.y));
      double2 d = csub(zk, zc);
      double2 od = make_double2(0.5 * d.y, -0.5 * d.x);  // (Z - conj Zc)/(2i)
      double2 f = cadd(e, cmul(w, od));
      emit(kk, f.x * s);
      emit(N - kk, f.y * s);
    };
#pragma unroll
    for (int m = 0; m < 4; m++) {
      const int k = t + m * TPV;
      if (k == 0) {
        double2 z0 = S[0];
        emit(0, (z0.x + z0.y) * s);
        emit(H, (z0.x - z0.y) * s);
      } else {
        const double2 w = __ldg(&tw[k]);
        pair_out(k, w);
        pair_out(H - k, make_double2(-w.x, w.y));
      }
    }
    if (t == 0) pair_out(H / 2, __ldg(&tw[H / 2]));  // k = H/2 pairs with itself
    if (SVF) {
      __syncthreads();
      constexpr int Q = (V * N) / NT;
      const double *O = Sd + 2 * V * VS;
#pragma unroll
      for (int q = 0; q < Q; q++) {
        int idx = threadIdx.x + q * NT;
        int vv = idx % V, k = idx / V;
        st(b, v0 + vv, k, O[2 * vv * VS + dpos(k)]);
      }
    }
  } else {
    // Hermitian -> Z (even/odd packing): thread t forms Z at k and H-k for
    // k = t + m*TPV (m < 4), thread 0 also k = H/2.
    auto X = [&](int j) -> double {
      if constexpr (NR > 0) return ld.staged(b, vg, j, Rw);
      else return LVF ? SdV[dpos(j)] : ld(b, vg, j);
    };
    double2 zp[9];
    int zk[9];
#pragma unroll
    for (int m = 0; m < 4; m++) {
      const int k = t + m * TPV;
      if (k == 0) {
        double F0 = X(0), Fh = X(H);
        zp[2 * m] = make_double2(0.5 * (F0 + Fh), 0.5 * (F0 - Fh));
        zk[2 * m] = 0;
        zk[2 * m + 1] = -1;
        zp[2 * m + 1] = make_double2(0.0, 0.0);
      } else {
        const double a = X(k), bq = X(N - k), c = X(H - k), dq = X(N - (H - k));
        const double2 wk = __ldg(&tw[k]);  // tw[H-k] = -conj(tw[k])
#pragma unroll
        for (int pass = 0; pass < 2; pass++) {
          const int kk = pass == 0 ? k : H - k;
          double2 F = pass == 0 ? make_double2(a, bq) : make_double2(c, dq);
          double2 G = pass == 0 ? make_double2(c, -dq) : make_double2(a, -bq);  // conj F(H-kk)
          double2 e = make_double2(0.5 * (F.x + G.x), 0.5 * (F.y + G.y));
          double2 d = make_double2(0.5 * (F.x - G.x), 0.5 * (F.y - G.y));
          const double2 w = pass == 0 ? wk : make_double2(-wk.x, wk.y);
          double2 o = cmul(d, cconj(w));
          zp[2 * m + pass] = make_double2(e.x - o.y, e.y + o.x);
          zk[2 * m + pass] = kk;
        }
      }
    }
    if (t == 0) {
      const int kk = H / 2;
      double2 F = make_double2(X(kk), X(N - kk));
      double2 G = make_double2(X(H - kk), -X(N - (H - kk)));
      double2 e = make_double2(0.5 * (F.x + G.x), 0.5 * (F.y + G.y));
      double2 d = make_double2(0.5 * (F.x - G.x), 0.5 * (F.y - G.y));
      double2 o = cmul(d, cconj(__ldg(&tw[kk])));
      zp[8] = make_double2(e.x - o.y, e.y + o.x);
      zk[8] = kk;
    } else {
      zk[8] = -1;
      zp[8] = make_double2(0.0, 0.0);
    }
    if (LVF || NR > 0) __syncthreads();  // staged input fully read before Z overwrites it
#pragma unroll
    for (int q = 0; q < 9; q++)
      if (zk[q] >= 0) S[cpad(zk[q])] = zp[q];
    __syncthreads();
#pragma unroll
    for (int m = 0; m < 8; m++) x[m] = S[cpad(t + m * TPV)];
    __syncthreads();
    rf_complex<LOGH, false>(x, S, t, tw, N);
    const double s = 2.0 / sqrt((double)N);
    if (!SVF) {
#pragma unroll
      for (int m = 0; m < 8; m++) {
        int e = t + m * TPV;
        if constexpr (has_pair<ST>::value) {
          st.pair(b, vg, 2 * e, make_double2(x[m].x * s, x[m].y * s));
        } else {
          st(b, vg, 2 * e, x[m].x * s);
          st(b, vg, 2 * e + 1, x[m].y * s);
        }
      }
    } else {
#pragma unroll
      for (int m = 0; m < 8; m++) S[cpad(t + m * TPV)] = x[m];
      __syncthreads();
      constexpr int Q = (V * N) / NT;
#pragma unroll
      for (int q = 0; q < Q; q++) {
        int idx = threadIdx.x + q * NT;
        int vv = idx % V, k = idx / V;
        st(b, v0 + vv, k, Sd[2 * vv * VS + dpos(k)] * s);
      }
    }
  }
}


}  // namespace casl
