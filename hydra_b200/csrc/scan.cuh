// Device-wide scans and a bump allocator over the handle's scratch arena.
//
// Scans are three-phase (per-block scan, scan of block totals in one block,
// carry add), deterministic, with 4096 elements per block.  Integer scans
// are exact; the segmented double scan sums in a fixed order (the same on
// every run), restarting at every head flag.
#pragma once

#include "common.cuh"
#include "state.cuh"

namespace casl {

// Bump allocator over one device buffer (256-byte aligned pieces).  Once a
// request does not fit, every later request fails too, so checking the last
// pointer of a group of requests checks them all.
struct Arena {
  char *base;
  size_t cap, off;
  bool failed = false;
  template <class T>
  T *get(size_t count) {
    size_t bytes = (count * sizeof(T) + 255) & ~(size_t)255;
    if (failed || base == nullptr || off + bytes > cap) {
      failed = true;
      return nullptr;
    }
    T *p = reinterpret_cast<T *>(base + off);
    off += bytes;
    return p;
  }
};

constexpr int SCAN_BLOCK = 1024;
constexpr int SCAN_ITEMS = 4;
constexpr int SCAN_TILE = SCAN_BLOCK * SCAN_ITEMS;

template <class T>
__device__ __forceinline__ T warp_incl_scan(T x) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    T y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  return x;
}

// Block-wide exclusive scan of one value per thread; returns the block total
// through *total.  blockDim.x must be SCAN_BLOCK.
template <class T>
__device__ T block_excl_scan(T v, T *total) {
  __shared__ T wsum[32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  T incl = warp_incl_scan(v);
  if (lane == 31) wsum[wid] = incl;
  __syncthreads();
  if (wid == 0) {
    T w = wsum[lane];
    T wi = warp_incl_scan(w);
    wsum[lane] = wi - w;
    if (lane == 31) *total = wi;
  }
  __syncthreads();
  T r = incl - v + wsum[wid];
  __syncthreads();
  return r;
}

// Block-wide exclusive scan for any block size (a multiple of 32).
template <class T>
__device__ T block_excl_scan_any(T v, T *total) {
  __shared__ T wsum[32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  T incl = warp_incl_scan(v);
  if (lane == 31) wsum[wid] = incl;
  __syncthreads();
  if (wid == 0) {
    T w = lane < nw ? wsum[lane] : T(0);
    T wi = warp_incl_scan(w);
    wsum[lane] = wi - w;
    if (lane == 31) *total = wi;
  }
  __syncthreads();
  T r = incl - v + wsum[wid];
  __syncthreads();
  return r;
}

template <class T>
__global__ void __launch_bounds__(SCAN_BLOCK) k_scan_tiles(const T *__restrict__ in,
                                                           T *__restrict__ out,
                                                           T *__restrict__ tile_tot, long long n) {
  CASL_PDL_ENTRY();
  __shared__ T tot;
  long long base = (long long)blockIdx.x * SCAN_TILE + (long long)threadIdx.x * SCAN_ITEMS;
  T v[SCAN_ITEMS];
  T s = 0;
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; k++) {
    v[k] = (base + k < n) ? in[base + k] : T(0);
    s += v[k];
  }
  T ex = block_excl_scan<T>(s, &tot);
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; k++) {
    if (base + k < n) out[base + k] = ex;
    ex += v[k];
  }
  if (threadIdx.x == 0) tile_tot[blockIdx.x] = tot;
}

// Exclusive scan of the tile totals in one block; writes the grand total.
template <class T>
__global__ void __launch_bounds__(SCAN_BLOCK) k_scan_totals(T *__restrict__ tot, int ntiles,
                                                            T *__restrict__ grand) {
  CASL_PDL_ENTRY();
  __shared__ T t;
  __shared__ T carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < ntiles; base += SCAN_BLOCK) {
    int i = base + threadIdx.x;
    T v = i < ntiles ? tot[i] : T(0);
    T ex = block_excl_scan<T>(v, &t);
    if (i < ntiles) tot[i] = ex + carry;
    __syncthreads();
    if (threadIdx.x == 0) carry += t;
    __syncthreads();
  }
  if (threadIdx.x == 0 && grand) *grand = carry;
}

template <class T>
__global__ void k_scan_add(T *__restrict__ out, const T *__restrict__ tot, long long n) {
  CASL_PDL_ENTRY();
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] += tot[i / SCAN_TILE];
}

// One block scans a small array tile by tile (one launch instead of three).
template <class T>
__global__ void __launch_bounds__(SCAN_BLOCK) k_scan_small(const T *__restrict__ in,
                                                           T *__restrict__ out, long long n,
                                                           T *__restrict__ grand) {
  CASL_PDL_ENTRY();
  __shared__ T tot;
  __shared__ T carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (long long tile = 0; tile * SCAN_TILE < n; tile++) {
    long long base = tile * SCAN_TILE + (long long)threadIdx.x * SCAN_ITEMS;
    T v[SCAN_ITEMS];
    T s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; k++) {
      v[k] = (base + k < n) ? in[base + k] : T(0);
      s += v[k];
    }
    T ex = block_excl_scan<T>(s, &tot) + carry;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; k++) {
      if (base + k < n) out[base + k] = ex;
      ex += v[k];
    }
    __syncthreads();
    if (threadIdx.x == 0) carry += tot;
    __syncthreads();
  }
  if (threadIdx.x == 0 && grand) *grand = carry;
}

// Two-pass scan for mid-size arrays: per-tile sums, then each tile adds the
// sum of the tiles before it (read by the tile's own block, so no third
// kernel) and scans itself.  VEC: items move as one 16-byte access per
// thread (in/out 16-byte aligned, 4-byte T).
template <class T, bool VEC>
__device__ __forceinline__ void scan_load(const T *__restrict__ in, long long base, long long n,
                                          T (&v)[SCAN_ITEMS]) {
  if (VEC && base + SCAN_ITEMS <= n) {
    int4 q = *reinterpret_cast<const int4 *>(in + base);
    v[0] = (T)q.x; v[1] = (T)q.y; v[2] = (T)q.z; v[3] = (T)q.w;
  } else {
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; k++) v[k] = (base + k < n) ? in[base + k] : T(0);
  }
}

template <class T, bool VEC>
__global__ void __launch_bounds__(SCAN_BLOCK) k_scan_tilesum(const T *__restrict__ in,
                                                             T *__restrict__ tile_tot, long long n) {
  CASL_PDL_ENTRY();
  __shared__ T part[32];
  long long base = (long long)blockIdx.x * SCAN_TILE + (long long)threadIdx.x * SCAN_ITEMS;
  T v[SCAN_ITEMS];
  scan_load<T, VEC>(in, base, n, v);
  T s = v[0] + v[1] + v[2] + v[3];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    T w = part[threadIdx.x];
    for (int o = 16; o > 0; o >>= 1) w += __shfl_down_sync(0xffffffffu, w, o);
    if (threadIdx.x == 0) tile_tot[blockIdx.x] = w;
  }
}

template <class T, bool VEC>
__global__ void __launch_bounds__(SCAN_BLOCK) k_scan_apply(const T *in, T *out,
                                                           const T *__restrict__ tile_tot,
                                                           long long n, T *__restrict__ grand) {
  CASL_PDL_ENTRY();
  __shared__ T part[32];
  __shared__ T tot;
  // offset of this tile: sum of the earlier tiles' totals (fixed order)
  T o = 0;
  for (int i = threadIdx.x; i < (int)blockIdx.x; i += SCAN_BLOCK) o += tile_tot[i];
  for (int d = 16; d > 0; d >>= 1) o += __shfl_down_sync(0xffffffffu, o, d);
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = o;
  __syncthreads();
  if (threadIdx.x < 32) {
    T w = part[threadIdx.x];
    for (int d = 16; d > 0; d >>= 1) w += __shfl_down_sync(0xffffffffu, w, d);
    if (threadIdx.x == 0) part[0] = w;
  }
  __syncthreads();
  const T off = part[0];
  __syncthreads();
  long long base = (long long)blockIdx.x * SCAN_TILE + (long long)threadIdx.x * SCAN_ITEMS;
  T v[SCAN_ITEMS];
  scan_load<T, VEC>(in, base, n, v);
  T ex = block_excl_scan<T>(v[0] + v[1] + v[2] + v[3], &tot) + off;
  T r[SCAN_ITEMS];
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; k++) {
    r[k] = ex;
    ex += v[k];
  }
  if (VEC && base + SCAN_ITEMS <= n) {
    *reinterpret_cast<int4 *>(out + base) = make_int4((int)r[0], (int)r[1], (int)r[2], (int)r[3]);
  } else {
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; k++)
      if (base + k < n) out[base + k] = r[k];
  }
  if (grand && blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) *grand = off + tot;
}

constexpr int SCAN_TWO_PASS_MAX_TILES = 8192;  // 33.5M elements; above, three phases

// out[i] = sum_{j<i} in[j]; *grand (device, optional) = sum of all.
// in and out may alias.  tmp needs ceil(n/SCAN_TILE) elements.
template <class T>
int exclusive_scan(cudaStream_t st, const T *in, T *out, long long n, T *tmp, T *grand) {
  if (n <= 0) {
    if (grand) cudaMemsetAsync(grand, 0, sizeof(T), st);
    return 0;
  }
  if (n <= 16 * SCAN_TILE) {
    CASL_K(k_scan_small<T>, 1, SCAN_BLOCK, 0, st)(in, out, n, grand);
    return (int)cudaGetLastError();
  }
  if ((n + SCAN_TILE - 1) / SCAN_TILE <= SCAN_TWO_PASS_MAX_TILES) {
    const int tiles = (int)((n + SCAN_TILE - 1) / SCAN_TILE);
    const bool vec = sizeof(T) == 4 && (((uintptr_t)in | (uintptr_t)out) & 15) == 0;
    if (vec) {
      CASL_K((k_scan_tilesum<T, true>), tiles, SCAN_BLOCK, 0, st)(in, tmp, n);
      CASL_K((k_scan_apply<T, true>), tiles, SCAN_BLOCK, 0, st)(in, out, tmp, n, grand);
    } else {
      CASL_K((k_scan_tilesum<T, false>), tiles, SCAN_BLOCK, 0, st)(in, tmp, n);
      CASL_K((k_scan_apply<T, false>), tiles, SCAN_BLOCK, 0, st)(in, out, tmp, n, grand);
    }
    return (int)cudaGetLastError();
  }
  int tiles = (int)((n + SCAN_TILE - 1) / SCAN_TILE);
  CASL_K(k_scan_tiles<T>, tiles, SCAN_BLOCK, 0, st)(in, out, tmp, n);
  CASL_K(k_scan_totals<T>, 1, SCAN_BLOCK, 0, st)(tmp, tiles, grand);
  CASL_K(k_scan_add<T>, (int)((n + 255) / 256), 256, 0, st)(out, tmp, n);
  return (int)cudaGetLastError();
}

inline long long scan_tmp_elems(long long n) { return (n + SCAN_TILE - 1) / SCAN_TILE + 1; }

// ---------------------------------------------------------------------------
// Segmented inclusive scan of doubles: out[i] = sum of in[j] for j from the
// last head at or before i through i.  head[i] != 0 starts a segment.
// ---------------------------------------------------------------------------
struct SegPair {
  double v;
  int f;
};
__device__ __forceinline__ SegPair seg_op(SegPair a, SegPair b) {
  SegPair r;
  r.f = a.f | b.f;
  r.v = b.f ? b.v : a.v + b.v;
  return r;
}
__device__ __forceinline__ SegPair warp_seg_incl(SegPair x) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    SegPair y;
    y.v = __shfl_up_sync(0xffffffffu, x.v, o);
    y.f = __shfl_up_sync(0xffffffffu, x.f, o);
    if (lane >= o) x = seg_op(y, x);
  }
  return x;
}
// Exclusive (prefix before this thread) segmented scan across the block.
static __device__ SegPair block_seg_excl(SegPair x, SegPair *total) {
  __shared__ double wv[32];
  __shared__ int wf[32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  SegPair incl = warp_seg_incl(x);
  SegPair ex;
  ex.v = __shfl_up_sync(0xffffffffu, incl.v, 1);
  ex.f = __shfl_up_sync(0xffffffffu, incl.f, 1);
  if (lane == 0) { ex.v = 0.0; ex.f = 0; }
  if (lane == 31) { wv[wid] = incl.v; wf[wid] = incl.f; }
  __syncthreads();
  if (wid == 0) {
    SegPair w{wv[lane], wf[lane]};
    SegPair wi = warp_seg_incl(w);
    SegPair we;
    we.v = __shfl_up_sync(0xffffffffu, wi.v, 1);
    we.f = __shfl_up_sync(0xffffffffu, wi.f, 1);
    if (lane == 0) { we.v = 0.0; we.f = 0; }
    wv[lane] = we.v;
    wf[lane] = we.f;
    if (lane == 31) *total = wi;
  }
  __syncthreads();
  SegPair pre{wv[wid], wf[wid]};
  SegPair r = seg_op(pre, ex);
  __syncthreads();
  return r;
}

static __global__ void __launch_bounds__(SCAN_BLOCK) k_segscan_tiles(const double *__restrict__ in,
                                                              const int *__restrict__ head,
                                                              double *__restrict__ out,
                                                              SegPair *__restrict__ tile_tot,
                                                              long long n) {
  CASL_PDL_ENTRY();
  __shared__ SegPair tot;
  long long base = (long long)blockIdx.x * SCAN_TILE + (long long)threadIdx.x * SCAN_ITEMS;
  SegPair loc[SCAN_ITEMS];
  SegPair acc{0.0, 0};
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; k++) {
    bool ok = base + k < n;
    loc[k].v = ok ? in[base + k] : 0.0;
    loc[k].f = ok ? (head[base + k] != 0) : 0;
    acc = seg_op(acc, loc[k]);
  }
  SegPair ex = block_seg_excl(acc, &tot);
  SegPair run = ex;
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; k++) {
    run = seg_op(run, loc[k]);
    if (base + k < n) out[base + k] = run.v;
  }
  if (threadIdx.x == 0) tile_tot[blockIdx.x] = tot;
}

// Exclusive segmented scan of tile totals (one block): carry into each tile.
static __global__ void __launch_bounds__(SCAN_BLOCK) k_segscan_totals(SegPair *__restrict__ tot,
                                                               int ntiles) {
  CASL_PDL_ENTRY();
  __shared__ SegPair t;
  __shared__ SegPair carry;
  if (threadIdx.x == 0) { carry.v = 0.0; carry.f = 0; }
  __syncthreads();
  for (int base = 0; base < ntiles; base += SCAN_BLOCK) {
    int i = base + threadIdx.x;
    SegPair v = i < ntiles ? tot[i] : SegPair{0.0, 0};
    SegPair ex = block_seg_excl(v, &t);
    SegPair c = carry;
    if (i < ntiles) tot[i] = seg_op(c, ex);
    __syncthreads();
    if (threadIdx.x == 0) carry = seg_op(carry, t);
    __syncthreads();
  }
}

// Add each tile's incoming carry to its elements before the tile's first head.
static __global__ void k_segscan_add(double *__restrict__ out, const int *__restrict__ head,
                              const SegPair *__restrict__ tot, long long n) {
  CASL_PDL_ENTRY();
  long long tile = blockIdx.x;
  long long beg = tile * SCAN_TILE, end = beg + SCAN_TILE < n ? beg + SCAN_TILE : n;
  double c = tot[tile].v;
  if (tile == 0) return;
  // elements up to (excluding) the first head of the tile receive the carry
  __shared__ long long first;
  if (threadIdx.x == 0) first = end;
  __syncthreads();
  for (long long i = beg + threadIdx.x; i < end; i += blockDim.x)
    if (head[i]) atomicMin((unsigned long long *)&first, (unsigned long long)i);
  __syncthreads();
  for (long long i = beg + threadIdx.x; i < first; i += blockDim.x) out[i] += c;
}

inline int segmented_scan(cudaStream_t st, const double *in, const int *head, double *out,
                          long long n, SegPair *tmp) {
  if (n <= 0) return 0;
  int tiles = (int)((n + SCAN_TILE - 1) / SCAN_TILE);
  CASL_K(k_segscan_tiles, tiles, SCAN_BLOCK, 0, st)(in, head, out, tmp, n);
  CASL_K(k_segscan_totals, 1, SCAN_BLOCK, 0, st)(tmp, tiles);
  CASL_K(k_segscan_add, tiles, 256, 0, st)(out, head, tmp, n);
  return (int)cudaGetLastError();
}

}  // namespace casl
