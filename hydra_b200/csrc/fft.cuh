// Batched real FFTs in the stafft "Hermitian" layout, one axis at a time.
//
// The transform restated (lib/stafft/stafft.f90:55-58,187-406):
//   forward:  X[k]   = Re F(k) / sqrt(n)   k = 0..n/2
//             X[n-k] = Im F(k) / sqrt(n)   k = 1..n/2-1,  F(k) = sum_j x_j e^{-2 pi i jk/n}
//   reverse:  the exact inverse.
// A 2-D ptospc/spctop (sta2dfft.f90:103-165) is two launches of this kernel,
// one per axis, with the transpose folded into the store/load addressing.
//
// B200 design: one CTA transforms V vectors of one field entirely in shared
// memory.  The real length-n transform runs as a complex length-n/2 Stockham
// FFT (radix 8, then 4 or 2) between two shared-memory buffers, bracketed by
// the even/odd untangling step.  Global traffic is exactly one read and one
// write of every element per axis; the load and store are functors so that
// pointwise spectral work (Green function, derivatives, filters, products)
// fuses into the transform instead of costing extra HBM passes.
#pragma once

#include "common.cuh"

namespace casl {

__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
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

// One Stockham pass of radix R over V complex vectors of length h held in
// `src` (vector stride ldc complex), writing `dst`.
template <int R, bool FWD>
__device__ __forceinline__ void stockham_pass(const double2 *src, double2 *dst, int V, int h, int ldc,
                                              int Ns, const double2 *__restrict__ tw, int n) {
  const int q = h / R;
  const int L = Ns * R;
  const int tstride = n / L;
  for (int w = threadIdx.x; w < V * q; w += blockDim.x) {
    int v = w / q, j = w - v * q;
    const double2 *s = src + v * ldc;
    double2 *d = dst + v * ldc;
    int k = j % Ns;
    double2 x[R];
#pragma unroll
    for (int r = 0; r < R; r++) x[r] = s[j + r * q];
    if (k) {
#pragma unroll
      for (int r = 1; r < R; r++) {
        double2 t = __ldg(&tw[r * k * tstride]);
        x[r] = cmul(x[r], FWD ? t : cconj(t));
      }
    }
    if (R == 8) dft8<FWD>(x);
    if (R == 4) dft4<FWD>(x[0], x[1], x[2], x[3]);
    if (R == 2) dft2<FWD>(x);
    int idxD = (j / Ns) * L + k;
#pragma unroll
    for (int r = 0; r < R; r++) d[idxD + r * Ns] = x[r];
  }
}

// Complex FFT of length h = 2^logh on V vectors, ping-ponging a <-> b.
// Returns the buffer holding the result.
template <bool FWD>
__device__ double2 *complex_fft(double2 *a, double2 *b, int V, int h, int ldc, int logh,
                                const double2 *__restrict__ tw, int n) {
  int Ns = 1;
  int rem = logh;
  while (rem > 0) {
    if (rem >= 3) {
      stockham_pass<8, FWD>(a, b, V, h, ldc, Ns, tw, n);
      Ns *= 8;
      rem -= 3;
    } else if (rem == 2) {
      stockham_pass<4, FWD>(a, b, V, h, ldc, Ns, tw, n);
      Ns *= 4;
      rem -= 2;
    } else {
      stockham_pass<2, FWD>(a, b, V, h, ldc, Ns, tw, n);
      Ns *= 2;
      rem -= 1;
    }
    __syncthreads();
    double2 *t = a;
    a = b;
    b = t;
  }
  return a;
}

// Plain strided load / store functors: element (b, v, j) at p[b*bs + v*vs + j*es].
struct LoadStrided {
  __host__ double bytes() const { return 8.0; }
  const double *p;
  long long bs, vs, es;
  __device__ __forceinline__ double operator()(int b, int v, int j) const {
    return p[b * bs + (long long)v * vs + (long long)j * es];
  }
};
struct StoreStrided {
  __host__ double bytes() const { return 8.0; }
  double *p;
  long long bs, vs, es;
  __device__ __forceinline__ void operator()(int b, int v, int k, double x) const {
    p[b * bs + (long long)v * vs + (long long)k * es] = x;
  }
};

// The kernel: grid (nvec / V, batch).  LVF / SVF: whether consecutive vectors
// (true) or consecutive elements (false) are adjacent in global memory for
// the load / the store, which sets the thread mapping for coalescing.
template <int V, bool FWD, bool LVF, bool SVF, class LD, class ST>
__global__ void __launch_bounds__(256) k_rfft(LD ld, ST st, const double2 *__restrict__ tw, int n,
                                              int logh) {
  extern __shared__ double2 smem[];
  const int h = n >> 1;
  const int ldc = h + 1;           // padded vector stride (complex units)
  const int ldr = 2 * ldc;         // same stride in doubles
  double2 *bufA = smem;
  double2 *bufB = smem + V * ldc;
  double *rA = reinterpret_cast<double *>(bufA);
  const int v0 = blockIdx.x * V;
  const int b = blockIdx.y;

  // Global -> shared, four independent loads in flight per thread.
  constexpr int U = 4;
  for (int base = threadIdx.x; base < V * n; base += U * blockDim.x) {
    double r[U];
    int off[U];
#pragma unroll
    for (int q = 0; q < U; q++) {
      int idx = base + q * blockDim.x;
      off[q] = -1;
      if (idx < V * n) {
        int v, j;
        if (LVF) { v = idx % V; j = idx / V; } else { v = idx / n; j = idx - (idx / n) * n; }
        r[q] = ld(b, v0 + v, j);
        off[q] = v * ldr + j;
      }
    }
#pragma unroll
    for (int q = 0; q < U; q++)
      if (off[q] >= 0) rA[off[q]] = r[q];
  }
  __syncthreads();

  if (FWD) {
    double2 *Z = complex_fft<true>(bufA, bufB, V, h, ldc, logh, tw, n);
    double *out = reinterpret_cast<double *>(Z == bufA ? bufB : bufA);
    const double s = 1.0 / sqrt((double)n);
    const int hh = h / 2;
    for (int w = threadIdx.x; w < V * (hh + 1); w += blockDim.x) {
      int v = w / (hh + 1), k = w - v * (hh + 1);
      const double2 *z = Z + v * ldc;
      double *o = out + v * ldr;
      if (k == 0) {
        double2 z0 = z[0];
        o[0] = (z0.x + z0.y) * s;
        o[h] = (z0.x - z0.y) * s;
      } else {
        // pair (k, h-k)
        for (int pass = 0; pass < 2; pass++) {
          int kk = pass == 0 ? k : h - k;
          if (pass == 1 && kk == k) break;
          double2 zk = z[kk], zc = cconj(z[h - kk]);
          double2 e = make_double2(0.5 * (zk.x + zc.x), 0.5 * (zk.y + zc.y));
          double2 d = csub(zk, zc);
          double2 od = make_double2(0.5 * d.y, -0.5 * d.x);  // (Z - conj Zc)/(2i)
          double2 f = cadd(e, cmul(__ldg(&tw[kk]), od));
          o[kk] = f.x * s;
          o[n - kk] = f.y * s;
        }
      }
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < V * n; idx += blockDim.x) {
      int v, k;
      if (SVF) { v = idx % V; k = idx / V; } else { v = idx / n; k = idx - (idx / n) * n; }
      st(b, v0 + v, k, out[v * ldr + k]);
    }
  } else {
    // Hermitian -> Z (even/odd packing), then inverse complex FFT.
    const int hh = h / 2;
    for (int w = threadIdx.x; w < V * (hh + 1); w += blockDim.x) {
      int v = w / (hh + 1), k = w - v * (hh + 1);
      const double *x = rA + v * ldr;
      double2 *z = bufB + v * ldc;
      if (k == 0) {
        double F0 = x[0], Fh = x[h];
        z[0] = make_double2(0.5 * (F0 + Fh), 0.5 * (F0 - Fh));
      } else {
        for (int pass = 0; pass < 2; pass++) {
          int kk = pass == 0 ? k : h - k;
          if (pass == 1 && kk == k) break;
          double2 F = make_double2(x[kk], x[n - kk]);
          double2 G = make_double2(x[h - kk], -x[n - (h - kk)]);  // conj F(h-kk)
          double2 e = make_double2(0.5 * (F.x + G.x), 0.5 * (F.y + G.y));
          double2 d = make_double2(0.5 * (F.x - G.x), 0.5 * (F.y - G.y));
          double2 o = cmul(d, cconj(__ldg(&tw[kk])));
          z[kk] = make_double2(e.x - o.y, e.y + o.x);
        }
      }
    }
    __syncthreads();
    double2 *Z = complex_fft<false>(bufB, bufA, V, h, ldc, logh, tw, n);
    const double *out = reinterpret_cast<const double *>(Z);
    const double s = 2.0 / sqrt((double)n);
    for (int idx = threadIdx.x; idx < V * n; idx += blockDim.x) {
      int v, k;
      if (SVF) { v = idx % V; k = idx / V; } else { v = idx / n; k = idx - (idx / n) * n; }
      st(b, v0 + v, k, out[v * ldr + k] * s);
    }
  }
}

inline size_t rfft_smem_bytes(int V, int n) { return (size_t)2 * V * (n / 2 + 1) * sizeof(double2); }

}  // namespace casl
