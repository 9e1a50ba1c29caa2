// The learned velocity closure: a small CNN that reads the coarse-grid PV and
// velocity of an inversion and predicts a correction to the velocity field
// that velint (contours.f90:136-169) interpolates bilinearly to the nodes.
//
// Network: four periodic 5x5 convolutions, 3 -> 32 -> 32 -> 32 -> 2 channels,
// GELU after the first three, BF16 weights and activations, FP32
// accumulation.  Every convolution -- forward, the input gradient and the
// weight gradient -- runs on the tensor cores (tcgen05.mma, accumulators in
// tensor memory), with its operands staged in shared memory by bulk copies.
//
// Activation layout ("padded planes"): a field of C channels on the n x n grid
// (rows = ix, columns = iy, the physical (ny,nx) order of the solver) is
// stored as [n+4 rows][C/8 planes][n+4 columns][8 channels] BF16, with a
// periodic halo of two rows and two columns on every side written by the
// kernel that produces the field.  One staged row segment of one plane is a
// contiguous run of 16-byte pixels, and the tap shift of the convolution along
// a row is a 16-byte step of the MMA operand's start address, so no im2col
// copy is needed: the 25 taps are 25 (or 50) MMAs over the same staged rows.
#include <cuda_bf16.h>
#include <limits.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <vector>

#include "state.cuh"
#include "tc.cuh"

namespace casl {
namespace net {

using bf16 = __nv_bfloat16;

constexpr int PAD = 2;          // halo rows / columns of the padded layout
constexpr int SEG = 128;        // output columns per CTA (the MMA's M)
constexpr int SEGIN = SEG + 4;  // staged input columns (two of halo each side)
constexpr int CS = SEGIN * 16;  // bytes of one staged row segment of one plane
constexpr int DZS = SEG * 16;   // bytes of one staged gradient row segment of one plane
enum { FWD_GELU = 0, FWD_LINEAR = 1, BWD_GELU = 2 };

// bf16 element offset of (row, col, 8-channel chunk) in the padded layout
__host__ __device__ __forceinline__ long long act_off(int n, int C, int row, int col, int chunk) {
  return ((((long long)(row + PAD) * (C / 8) + chunk) * (n + 2 * PAD)) + (col + PAD)) * 8;
}
inline long long act_elems(int n, int C) { return (long long)(n + 2 * PAD) * (n + 2 * PAD) * C; }

__device__ __forceinline__ float gelu_f(float x) {
  return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f));
}
__device__ __forceinline__ float gelu_d(float x) {
  return 0.5f * (1.0f + erff(x * 0.70710678118654752f)) +
         x * 0.39894228040143268f * expf(-0.5f * x * x);
}

__device__ __forceinline__ uint4 pack8(const float *v) {
  uint4 u;
  __nv_bfloat162 h;
  h = __floats2bfloat162_rn(v[0], v[1]); u.x = *reinterpret_cast<uint32_t *>(&h);
  h = __floats2bfloat162_rn(v[2], v[3]); u.y = *reinterpret_cast<uint32_t *>(&h);
  h = __floats2bfloat162_rn(v[4], v[5]); u.z = *reinterpret_cast<uint32_t *>(&h);
  h = __floats2bfloat162_rn(v[6], v[7]); u.w = *reinterpret_cast<uint32_t *>(&h);
  return u;
}
__device__ __forceinline__ void unpack8(uint4 u, float *v) {
  const uint32_t w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
  for (int i = 0; i < 4; i++) {
    __nv_bfloat162 h = *reinterpret_cast<const __nv_bfloat162 *>(&w[i]);
    float2 f = __bfloat1622float2(h);
    v[2 * i] = f.x;
    v[2 * i + 1] = f.y;
  }
}

// Stores the C channels of pixel (row, col) and its periodic halo copies.
template <int C>
__device__ __forceinline__ void store_px(bf16 *buf, int n, int row, int col, const float *v) {
  int rr[2] = {row, row < PAD ? row + n : (row >= n - PAD ? row - n : INT_MIN)};
  int cc[2] = {col, col < PAD ? col + n : (col >= n - PAD ? col - n : INT_MIN)};
#pragma unroll
  for (int c = 0; c < C / 8; c++) {
    const uint4 pk = pack8(v + 8 * c);
#pragma unroll
    for (int a = 0; a < 2; a++)
#pragma unroll
      for (int b = 0; b < 2; b++)
        if (rr[a] != INT_MIN && cc[b] != INT_MIN)
          *reinterpret_cast<uint4 *>(buf + act_off(n, C, rr[a], cc[b], c)) = pk;
  }
}

// ---------------------------------------------------------------------------
// Convolution (forward, or input gradient with the flipped weights)
// ---------------------------------------------------------------------------
struct ConvArgs {
  const bf16 *in;     // CIN channels, padded layout
  const bf16 *wimg;   // [5 kx][CIN/8][5 (4-ky)][COUT][8]: the shared-memory image of the weights
  const float *bias;  // FWD modes: COUT entries
  bf16 *out;          // FWD_GELU / BWD_GELU: COUT channels, padded layout
  bf16 *zout;         // FWD_GELU: pre-activations (nullable)
  const bf16 *zprev;  // BWD_GELU: pre-activations of the layer below (COUT channels)
  float *fout;        // FWD_LINEAR: [cout_real][n][n]
  float *dbias;       // BWD_GELU: += sum over pixels of the stored gradient (nullable)
  int n, cout_real;
  int *err;
};

template <int CIN, int COUT, int R>
struct ConvSmem {
  static constexpr int RS = (CIN / 8) * CS;            // one staged row, all planes
  static constexpr int IN_BYTES = (R + 4) * RS;        // one tile's input rows
  static constexpr int W_BYTES = 25 * (CIN / 8) * COUT * 16;
  static constexpr int BAR_OFF = W_BYTES + 2 * IN_BYTES;  // weights, two input buffers
  static constexpr int TOTAL = BAR_OFF + 80;
  static constexpr int ACC = R * COUT;                 // TMEM columns of one tile
  static constexpr int TCOLS = 2 * ACC < 32 ? 32 : 2 * ACC;
  static_assert(TCOLS <= 512 && (TCOLS & (TCOLS - 1)) == 0, "TMEM columns");
  static_assert(CIN % 16 == 0 && COUT % 16 == 0 && COUT <= 32, "channel counts");
  static_assert(R % 2 == 0, "rows split between two warp halves");
};

// A persistent CTA per SM walks a list of tiles (128 output columns x R
// rows; tile j: column strip j % (n/128), rows (j / (n/128)) * R ...).
// Warp-specialised: the last warp (one thread) stages the weight image once and
// each tile's input rows by bulk copies into one of two buffers, and issues
// the tile's MMAs into one of two TMEM accumulators; the others drain the
// accumulators (bias, GELU, stores) and clear them.  Barriers, not block
// syncs, couple them: full[b] (rows of buffer b arrived), mdone[b] (MMAs
// into accumulator b complete, which also frees input buffer b) and
// afree[b] (accumulator b drained and cleared), so the tensor core, the
// copy engine and the epilogue warps all run at once.  Within a tile,
// staged input row i (global row y0+i-2) feeds output rows r = i-4 .. i
// (those inside the tile) through tap row ky = i - r: one MMA per (i, kx,
// plane pair) with A[m][k] = input(row y0+i-2, column x0+m+kx-2, channel k
// of the pair) and B the weights of all those rows' ky stacked along N --
// the image keeps ky descending so that ascending output rows (ascending
// TMEM columns) meet their ky in order.  TMEM lane m is output column x0+m;
// row r's COUT accumulators are columns [r*COUT, (r+1)*COUT) of the tile's
// accumulator.  Epilogue warp w drains lanes 32(w%4).. of rows r = w/4,
// w/4 + EPI/4, ...  Every wait is bounded: one that gives up sets CASL_ETIMEOUT
// and stops the CTA once the copies and MMAs it issued have completed (again
// bounded).
// Epilogue warps: four per row of a tile in the forward modes (one row
// each); the input-gradient mode, whose epilogue holds more registers, uses
// half as many, two rows each.
template <int R, int MODE>
constexpr int conv_epi_warps() { return MODE == BWD_GELU ? 2 * R : 4 * R; }
template <int R, int MODE>
constexpr int conv_threads() { return 32 * (conv_epi_warps<R, MODE>() + 1); }

template <int CIN, int COUT, int R, int MODE>
__global__ void __launch_bounds__(conv_threads<R, MODE>(), 1) k_conv5(ConvArgs a) {
  constexpr int EPI = conv_epi_warps<R, MODE>();
  using S = ConvSmem<CIN, COUT, R>;
  extern __shared__ __align__(128) unsigned char smem[];
  unsigned char *w_s = smem;
  unsigned char *in_s0 = smem + S::W_BYTES;
  // barriers: [0] weights, [1 + b] full, [3 + b] mdone, [5 + b] afree
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem + S::BAR_OFF);
  uint32_t *tslot = reinterpret_cast<uint32_t *>(bars + 7);
  volatile int *abort_s = reinterpret_cast<volatile int *>(tslot + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int n = a.n;
  const int nstrip = n / SEG, ntiles = nstrip * (n / R);
  const int G = gridDim.x;
  CASL_PDL_ENTRY();
  if (tid == 0) {
    for (int q = 0; q < 5; q++) tc::mbar_init(&bars[q], 1);
    tc::mbar_init(&bars[5], EPI);
    tc::mbar_init(&bars[6], EPI);
    tc::mbar_fence_init();
    *abort_s = 0;
  }
  __syncthreads();
  if (warp == 0) tc::tmem_alloc(tslot, S::TCOLS);
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tbase = *tslot;
  const uint32_t lane_base = (uint32_t)(32 * (warp & 3)) << 16;
  // every MMA accumulates: clear both accumulators (warps 0-3 hold the 128 lanes)
  if (warp < 4)
    for (int c0 = 0; c0 < S::TCOLS; c0 += 32) tc::tmem_zero32(tbase + lane_base + (uint32_t)c0);
  tc::tmem_wait_st();
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const int ntile_cta = blockIdx.x < ntiles ? (ntiles - 1 - blockIdx.x) / G + 1 : 0;
  if (warp == EPI) {
    if (lane == 0) {
      // tile t's R+4 input rows (all planes) into buffer t & 1
      auto load_tile = [&](int t) {
        const int j = blockIdx.x + t * G, b = t & 1;
        const int x0 = (j % nstrip) * SEG, y0 = (j / nstrip) * R;
        unsigned char *dst = in_s0 + b * S::IN_BYTES;
        tc::mbar_expect_tx(&bars[1 + b], S::IN_BYTES);
        for (int i = 0; i < R + 4; i++)
          for (int c = 0; c < CIN / 8; c++)
            tc::bulk_g2s(dst + i * S::RS + c * CS, a.in + act_off(n, CIN, y0 - 2 + i, x0 - 2, c),
                         CS, &bars[1 + b]);
      };
      tc::mbar_expect_tx(&bars[0], S::W_BYTES);
      tc::bulk_g2s(w_s, a.wimg, S::W_BYTES, &bars[0]);
      if (ntile_cta > 0) load_tile(0);
      int loaded = ntile_cta > 0 ? 1 : 0, issued = 0;  // tiles loaded / with MMAs issued
      bool ok = tc::mbar_wait(&bars[0], 0);
      for (int t = 0; ok && t < ntile_cta; t++) {
        const int b = t & 1;
        // rows of tile t, accumulator b drained (tile t-2)
        ok = tc::mbar_wait(&bars[1 + b], (t >> 1) & 1);
        if (ok && t >= 2) ok = tc::mbar_wait(&bars[5 + b], ((t - 2) >> 1) & 1);
        if (!ok || *abort_s) break;
        tc::tc_fence_after();
        const uint32_t in_a = tc::smem_u32(in_s0 + b * S::IN_BYTES), w_a = tc::smem_u32(w_s);
        const uint32_t acc = tbase + (uint32_t)(b * S::ACC);
        for (int i = 0; i < R + 4; i++) {
          const int r_lo = i - 4 > 0 ? i - 4 : 0, r_hi = i < R - 1 ? i : R - 1;
          const int nrow = r_hi - r_lo + 1, ky_hi = i - r_lo;
          const uint32_t idesc = tc::idesc_bf16(128, nrow * COUT, false, false);
          for (int kx = 0; kx < 5; kx++)
#pragma unroll
            for (int cp = 0; cp < CIN / 16; cp++) {
              const uint64_t ad = tc::sdesc(in_a + i * S::RS + 2 * cp * CS + kx * 16, CS, 128);
              const uint64_t bd =
                  tc::sdesc(w_a + ((kx * (CIN / 8) + 2 * cp) * 5 + (4 - ky_hi)) * COUT * 16,
                            5 * COUT * 16, 128);
              tc::mma_bf16(acc + (uint32_t)(r_lo * COUT), ad, bd, idesc, 1u);
            }
        }
        tc::mma_commit(&bars[3 + b]);
        issued = t + 1;
        // tile t+1's rows into the other buffer once tile t-1's MMAs (its
        // readers) have completed
        if (t + 1 < ntile_cta) {
          if (t >= 1) ok = tc::mbar_wait(&bars[3 + (b ^ 1)], ((t - 1) >> 1) & 1);
          if (!ok) break;
          load_tile(t + 1);
          loaded = t + 2;
        }
      }
      if (!ok) {
        *abort_s = 1;
        atomicExch(a.err, CASL_ETIMEOUT);
      }
      // before the CTA ends: the last copies and MMAs issued have landed
      if (loaded > issued && loaded >= 1) {
        const int t = loaded - 1;
        tc::mbar_wait(&bars[1 + (t & 1)], (t >> 1) & 1);
      }
      if (issued >= 1) {
        const int t = issued - 1;
        tc::mbar_wait(&bars[3 + (t & 1)], (t >> 1) & 1);
      }
    }
  } else {
    float dsum[COUT];
#pragma unroll
    for (int co = 0; co < COUT; co++) dsum[co] = 0.0f;
    const int r0 = warp >> 2;  // this warp's rows: r0, r0 + EPI/4, ...
    for (int t = 0; t < ntile_cta; t++) {
      const int b = t & 1;
      const bool okp = !*abort_s && tc::mbar_wait(&bars[3 + b], (t >> 1) & 1);
      tc::tc_fence_after();
      if (!okp) {
        *abort_s = 1;
        atomicExch(a.err, CASL_ETIMEOUT);
        break;
      }
      const int j = blockIdx.x + t * G;
      const int x0 = (j % nstrip) * SEG, y0 = (j / nstrip) * R;
      const int col = x0 + (warp & 3) * 32 + lane;
      for (int r = r0; r < R; r += EPI / 4) {
        const int row = y0 + r;
        float v[COUT];
        const uint32_t taddr = tbase + lane_base + (uint32_t)(b * S::ACC + r * COUT);
        if (COUT == 32) {
          tc::tmem_ld32(taddr, v);
          tc::tmem_zero32(taddr);
        } else {
          tc::tmem_ld16(taddr, v);
          tc::tmem_zero16(taddr);
        }
        if (MODE == FWD_LINEAR) {
          for (int co = 0; co < a.cout_real; co++)
            a.fout[((long long)co * n + row) * n + col] = v[co] + a.bias[co];
        } else if (MODE == FWD_GELU) {
#pragma unroll
          for (int co = 0; co < COUT; co++) v[co] += a.bias[co];
          if (a.zout) store_px<COUT>(a.zout, n, row, col, v);
#pragma unroll
          for (int co = 0; co < COUT; co++) v[co] = gelu_f(v[co]);
          store_px<COUT>(a.out, n, row, col, v);
        } else {
#pragma unroll
          for (int c = 0; c < COUT / 8; c++) {
            float z[8];
            unpack8(*reinterpret_cast<const uint4 *>(a.zprev + act_off(n, COUT, row, col, c)), z);
#pragma unroll
            for (int e = 0; e < 8; e++) {
              const float g = v[8 * c + e] * gelu_d(z[e]);
              const float gr = __bfloat162float(__float2bfloat16_rn(g));
              v[8 * c + e] = gr;
              dsum[8 * c + e] += gr;
            }
          }
          store_px<COUT>(a.out, n, row, col, v);
        }
      }
      // accumulator b drained and cleared: one arrival per warp
      tc::tmem_wait_st();
      tc::tc_fence_before();
      __syncwarp();
      if (lane == 0) tc::mbar_arrive(&bars[5 + b]);
    }
    if (MODE == BWD_GELU && a.dbias) {
#pragma unroll
      for (int co = 0; co < COUT; co++) {
        float s = dsum[co];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0 && s != 0.0f) atomicAdd(&a.dbias[co], s);
      }
    }
  }
  tc::tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc::tc_fence_after();
    tc::tmem_dealloc(tbase, S::TCOLS);
  }
}

// ---------------------------------------------------------------------------
// Weight gradient
// ---------------------------------------------------------------------------
struct WgradArgs {
  const bf16 *in;  // layer input, CIN channels, padded layout
  const bf16 *dz;  // gradient of the layer's pre-activation, COUT channels, padded layout
  float *dw;       // += [25 taps][CIN][COUT]
  int n;
  int *err;
};

template <int CIN, int COUT, int R>
struct WgSmem {
  static constexpr int KYG = 128 / CIN;            // input rows one M = 128 operand spans
  static constexpr int NH = (5 + KYG - 1) / KYG;   // operands per (kx, K step)
  static constexpr int ROWS = R + NH * KYG - 1;    // staged rows (the last NH*KYG-5 zero)
  static constexpr int RS = (CIN / 8) * CS;
  static constexpr int IN_BYTES = ROWS * RS;
  static constexpr int RSZ = (COUT / 8) * DZS;
  static constexpr int DZ_BYTES = R * RSZ;
  static constexpr int TOTAL = IN_BYTES + DZ_BYTES + 64;
  static constexpr int NACC = 5 * NH * COUT;
  static constexpr int TCOLS = NACC <= 128 ? 128 : (NACC <= 256 ? 256 : 512);
  static_assert(NACC <= 512, "TMEM columns");
};

// dW(ky,kx)[ci][co] = sum over pixels of input(row+ky-2, col+kx-2, ci) *
// dz(row, col, co).  One CTA: columns [x0, x0+128) of rows [y0, y0+R).  The
// M = 128 rows of one MMA are (ky, ci) pairs of 128/CIN consecutive input
// rows -- staged rows are contiguous, so their planes are equally spaced and
// one MN-major operand spans them -- and K = 16 pixels per MMA; the tap shift
// kx is again a 16-byte step of the start address.  Accumulator (kx, h)
// holds ky = h*KYG .. h*KYG+KYG-1 (rows with ky > 4 are discarded).
template <int CIN, int COUT, int R>
__global__ void __launch_bounds__(128, 1) k_conv5_wgrad(WgradArgs a) {
  using S = WgSmem<CIN, COUT, R>;
  extern __shared__ __align__(128) unsigned char smem[];
  unsigned char *in_s = smem;
  unsigned char *dz_s = smem + S::IN_BYTES;
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem + S::IN_BYTES + S::DZ_BYTES);
  uint32_t *tslot = reinterpret_cast<uint32_t *>(bars + 2);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int n = a.n;
  const int x0 = blockIdx.x * SEG, y0 = blockIdx.y * R;
  CASL_PDL_ENTRY();
  if (tid == 0) {
    tc::mbar_init(&bars[0], 1);
    tc::mbar_init(&bars[1], 1);
    tc::mbar_fence_init();
  }
  // the staged rows past the real ones are read by discarded accumulator rows only
  for (int i = (R + 4) * S::RS / 16 + tid; i < S::IN_BYTES / 16; i += blockDim.x)
    reinterpret_cast<uint4 *>(in_s)[i] = make_uint4(0, 0, 0, 0);
  tc::fence_proxy_async_smem();
  __syncthreads();
  if (warp == 0) tc::tmem_alloc(tslot, S::TCOLS);
  if (tid == 0) {
    tc::mbar_expect_tx(&bars[0], (R + 4) * S::RS + S::DZ_BYTES);
    for (int i = 0; i < R + 4; i++)
      for (int c = 0; c < CIN / 8; c++)
        tc::bulk_g2s(in_s + i * S::RS + c * CS, a.in + act_off(n, CIN, y0 - 2 + i, x0 - 2, c), CS,
                     &bars[0]);
    for (int r = 0; r < R; r++)
      for (int c = 0; c < COUT / 8; c++)
        tc::bulk_g2s(dz_s + r * S::RSZ + c * DZS, a.dz + act_off(n, COUT, y0 + r, x0, c), DZS,
                     &bars[0]);
  }
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tbase = *tslot;
  bool ok = tc::mbar_wait(&bars[0], 0);
  if (tid == 0 && ok) {
    const uint32_t in_a = tc::smem_u32(in_s), dz_a = tc::smem_u32(dz_s);
    constexpr uint32_t IDESC = tc::idesc_bf16(128, COUT, true, true);
    for (int r = 0; r < R; r++)
      for (int kx = 0; kx < 5; kx++)
        for (int h = 0; h < S::NH; h++)
#pragma unroll
          for (int ks = 0; ks < SEG / 16; ks++) {
            const uint64_t ad =
                tc::sdesc(in_a + (r + h * S::KYG) * S::RS + kx * 16 + ks * 256, 128, CS);
            const uint64_t bd = tc::sdesc(dz_a + r * S::RSZ + ks * 256, 128, DZS);
            tc::mma_bf16(tbase + (kx * S::NH + h) * COUT, ad, bd, IDESC,
                         (r | ks) != 0 ? 1u : 0u);
          }
    tc::mma_commit(&bars[1]);
  }
  ok = ok && tc::mbar_wait(&bars[1], 0);
  tc::tc_fence_after();
  if (!ok) {
    if (lane == 0) atomicExch(a.err, CASL_ETIMEOUT);
  } else {
    const int m = warp * 32 + lane;
    const int g = m >> 3, e = m & 7;
    const int kyl = g / (CIN / 8), ci = (g % (CIN / 8)) * 8 + e;
    for (int kx = 0; kx < 5; kx++)
      for (int h = 0; h < S::NH; h++) {
        float v[COUT];
        const uint32_t taddr =
            tbase + ((uint32_t)(warp * 32) << 16) + (uint32_t)((kx * S::NH + h) * COUT);
        if (COUT == 32)
          tc::tmem_ld32(taddr, v);
        else
          tc::tmem_ld16(taddr, v);
        const int ky = h * S::KYG + kyl;
        if (ky < 5) {
          float *dst = a.dw + ((long long)(ky * 5 + kx) * CIN + ci) * COUT;
#pragma unroll
          for (int co = 0; co < COUT; co++) atomicAdd(dst + co, v[co]);
        }
      }
  }
  tc::tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc::tc_fence_after();
    tc::tmem_dealloc(tbase, S::TCOLS);
  }
}

// ---------------------------------------------------------------------------
// Layer table, parameters, weight images
// ---------------------------------------------------------------------------
constexpr int NL = 4;
// The network's output is the velocity correction on a grid SUB times as
// fine as the inversion's, as SUB x SUB sub-cells per coarse cell: channel
// comp*SUB^2 + a*SUB + b holds component comp (0: u, 1: v) at the point
// (SUB ix + a, SUB iy + b) of the fine grid.  A correction on the coarse
// grid itself cannot do better than about 1.1e-3 relative at 512^2 (the
// least-squares optimum of any coarse field under velint's bilinear
// interpolation), since the error is mostly the interpolation's own.
constexpr int SUB = 2;
constexpr int NOUT = 2 * SUB * SUB;
constexpr int OUTP = NOUT <= 16 ? 16 : 32;  // the output channels the MMAs run
static_assert(NOUT <= 32, "output channels");
constexpr int HID = 16;  // hidden channels
// Input channels: the coarse contour PV, u and v of the inversion, and the
// deviations of the fine (4n) contour levels at the 3 x 3 points (4cx +
// 2a - 2, 4cy + 2b - 2) of each coarse cell from the cell's weighted mean
// (the sub-cell shape of the contours that the coarse PV smooths away).
constexpr int NSUBF = 9;
constexpr int NIN = 3 + NSUBF;
static_assert(NIN <= 16, "input channels");
// real channel counts NIN -> HID -> HID -> HID -> NOUT, padded to the MMA's multiples of 16
__host__ __device__ constexpr int cin_r(int l) { return l == 0 ? NIN : HID; }
__host__ __device__ constexpr int cout_r(int l) { return l == NL - 1 ? NOUT : HID; }
__host__ __device__ constexpr int cin_p(int l) { return l == 0 ? 16 : HID; }
__host__ __device__ constexpr int cout_p(int l) { return l == NL - 1 ? OUTP : HID; }

struct ParamMap {
  int offw[NL], offb[NL], total;
};
inline ParamMap param_map() {
  ParamMap m{};
  int o = 0;
  for (int l = 0; l < NL; l++) {
    m.offw[l] = o;
    o += cout_r(l) * cin_r(l) * 25;
    m.offb[l] = o;
    o += cout_r(l);
  }
  m.total = o;
  return m;
}

struct LayerDev {
  bf16 *wf;     // forward image [25][CINP/8][COUTP][8]
  bf16 *wb;     // input-gradient image [25][COUTP/8][CINP][8] (flipped taps)
  float *bias;  // COUTP
  float *dw;    // [25][CINP][COUTP]
  float *db;    // COUTP
};

struct Params {
  const float *w;
  ParamMap m;
  LayerDev L[NL];
};

// Both weight images of every layer from the FP32 master parameters
// (W[co][ci][ky][kx], then b[co], layer after layer).
__global__ void k_weight_images(Params P) {
  CASL_PDL_ENTRY();
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (int l = 0; l < NL; l++) {
    const int ci_p = cin_p(l), co_p = cout_p(l), ci_r = cin_r(l), co_r = cout_r(l);
    const float *W = P.w + P.m.offw[l];
    const long long nimg = 25LL * ci_p * co_p;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nimg; t += stride) {
      // forward image: t = (((kx*(ci_p/8) + c)*5 + kyd)*co_p + co)*8 + e with
      // ci = 8c + e and ky = 4 - kyd
      {
        const int e = (int)(t % 8), co = (int)((t / 8) % co_p);
        const int kyd = (int)((t / 8 / co_p) % 5), c = (int)((t / 8 / co_p / 5) % (ci_p / 8));
        const int kx = (int)(t / 8 / co_p / 5 / (ci_p / 8));
        const int ci = 8 * c + e, tap = (4 - kyd) * 5 + kx;
        const float v = (ci < ci_r && co < co_r) ? W[(co * ci_r + ci) * 25 + tap] : 0.0f;
        P.L[l].wf[t] = __float2bfloat16_rn(v);
      }
      // input-gradient image (the convolution of the output gradient with the
      // taps flipped and ci, co exchanged): t = (((kx'*(co_p/8) + c')*5 + kyd')*ci_p
      // + ci)*8 + e with co = 8c' + e, ky' = 4 - kyd', tap = (4-ky')*5 + (4-kx')
      {
        const int e = (int)(t % 8), ci = (int)((t / 8) % ci_p);
        const int kyd = (int)((t / 8 / ci_p) % 5), c = (int)((t / 8 / ci_p / 5) % (co_p / 8));
        const int kxp = (int)(t / 8 / ci_p / 5 / (co_p / 8));
        const int co = 8 * c + e, tap = kyd * 5 + (4 - kxp);
        const float v = (ci < ci_r && co < co_r) ? W[(co * ci_r + ci) * 25 + tap] : 0.0f;
        P.L[l].wb[t] = __float2bfloat16_rn(v);
      }
    }
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < co_p; t += stride)
      P.L[l].bias[t] = t < co_r ? P.w[P.m.offb[l] + t] : 0.0f;
  }
}

// Flat FP32 gradient (the parameter order) from the per-layer accumulators.
__global__ void k_gather_grad(Params P, float *grad) {
  CASL_PDL_ENTRY();
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < P.m.total; i += stride) {
    int l = NL - 1;
    while (l > 0 && i < P.m.offw[l]) l--;
    const long long j = i - P.m.offw[l];
    const int ci_r = cin_r(l), co_r = cout_r(l);
    if (j < (long long)co_r * ci_r * 25) {
      const int tap = (int)(j % 25), ci = (int)((j / 25) % ci_r), co = (int)(j / 25 / ci_r);
      grad[i] = P.L[l].dw[((long long)tap * cin_p(l) + ci) * cout_p(l) + co];
    } else {
      grad[i] = P.L[l].db[j - (long long)co_r * ci_r * 25];
    }
  }
}

// Adam (Kingma & Ba 2015) on the FP32 master parameters, gradient taken from
// the per-layer accumulators: m = b1 m + (1-b1) g, v = b2 v + (1-b2) g^2,
// w -= lr * (m / (1-b1^t)) / (sqrt(v / (1-b2^t)) + eps).
__global__ void k_adam(Params P, float *w, float *mo, float *vo, float lr, float b1, float b2,
                       float eps, float c1, float c2) {
  CASL_PDL_ENTRY();
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < P.m.total; i += stride) {
    int l = NL - 1;
    while (l > 0 && i < P.m.offw[l]) l--;
    const long long j = i - P.m.offw[l];
    const int ci_r = cin_r(l), co_r = cout_r(l);
    float g;
    if (j < (long long)co_r * ci_r * 25) {
      const int tap = (int)(j % 25), ci = (int)((j / 25) % ci_r), co = (int)(j / 25 / ci_r);
      g = P.L[l].dw[((long long)tap * cin_p(l) + ci) * cout_p(l) + co];
    } else {
      g = P.L[l].db[j - (long long)co_r * ci_r * 25];
    }
    const float m = b1 * mo[i] + (1.0f - b1) * g;
    const float v = b2 * vo[i] + (1.0f - b2) * g * g;
    mo[i] = m;
    vo[i] = v;
    w[i] -= lr * (m / c1) / (sqrtf(v / c2) + eps);
  }
}

// FP32 channel-major input [3][n][n] -> padded 16-channel planes (13 zero).
__global__ void k_pack_input(const float *__restrict__ x, bf16 *__restrict__ x0, int n, int cin) {
  CASL_PDL_ENTRY();
  const long long nn = (long long)n * n;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nn;
       t += (long long)gridDim.x * blockDim.x) {
    const int row = (int)(t / n), col = (int)(t % n);
    float v[16];
#pragma unroll
    for (int c = 0; c < 16; c++) v[c] = c < cin ? x[c * nn + t] : 0.0f;
    store_px<16>(x0, n, row, col, v);
  }
}

// FP32 [cout][n][n] output gradient -> padded 16-channel planes, and its sum
// over pixels (the last layer's bias gradient).
template <int C>
__global__ void k_pack_grad(const float *__restrict__ g, bf16 *__restrict__ dz, int n, int cout,
                            float *__restrict__ db) {
  CASL_PDL_ENTRY();
  const long long nn = (long long)n * n;
  float sum[C];
#pragma unroll
  for (int c = 0; c < C; c++) sum[c] = 0.0f;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nn;
       t += (long long)gridDim.x * blockDim.x) {
    const int row = (int)(t / n), col = (int)(t % n);
    float v[C];
#pragma unroll
    for (int c = 0; c < C; c++) {
      v[c] = c < cout ? __bfloat162float(__float2bfloat16_rn(g[c * nn + t])) : 0.0f;
      sum[c] += v[c];
    }
    store_px<C>(dz, n, row, col, v);
  }
#pragma unroll
  for (int c = 0; c < C; c++) {
    float x = sum[c];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if ((threadIdx.x & 31) == 0 && c < cout) atomicAdd(&db[c], x);
  }
}

// ---------------------------------------------------------------------------
// Launches
// ---------------------------------------------------------------------------
constexpr int RF = 4;  // output rows per tile of the convolutions
constexpr int RW = 8;  // gradient rows per CTA of the weight gradients

template <int CIN, int COUT, int MODE>
static int launch_conv(const ConvArgs &a, cudaStream_t st) {
  using S = ConvSmem<CIN, COUT, RF>;
  auto k = k_conv5<CIN, COUT, RF, MODE>;
  static bool set = false;  // one per instance
  if (!set) {
    if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, S::TOTAL) !=
        cudaSuccess)
      return CASL_ECUDA;
    set = true;
  }
  // named by its template arguments for the per-launch timing report
  static char name[48];
  if (!name[0]) snprintf(name, sizeof name, "k_conv5<%d, %d, %d, %d>", CIN, COUT, RF, MODE);
  // persistent: one CTA per SM (at most one per tile)
  const int ntiles = (a.n / SEG) * (a.n / RF);
  const dim3 grid(ntiles < 148 ? ntiles : 148);
  constexpr int NT = conv_threads<RF, MODE>();
  for (bool once = kt_begin(name, grid, NT, S::TOTAL, st); once; once = kt_end())
    launch_of(k, grid, NT, S::TOTAL, st)(a);
  return cudaPeekAtLastError() == cudaSuccess ? CASL_OK : CASL_ECUDA;
}

template <int CIN, int COUT>
static int launch_wgrad(const WgradArgs &a, cudaStream_t st) {
  using S = WgSmem<CIN, COUT, RW>;
  auto k = k_conv5_wgrad<CIN, COUT, RW>;
  static bool set = false;
  if (!set) {
    if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, S::TOTAL) !=
        cudaSuccess)
      return CASL_ECUDA;
    set = true;
  }
  static char name[48];
  if (!name[0]) snprintf(name, sizeof name, "k_conv5_wgrad<%d, %d, %d>", CIN, COUT, RW);
  const dim3 grid(a.n / SEG, a.n / RW);
  for (bool once = kt_begin(name, grid, 128, S::TOTAL, st); once; once = kt_end())
    launch_of(k, grid, 128, S::TOTAL, st)(a);
  return cudaPeekAtLastError() == cudaSuccess ? CASL_OK : CASL_ECUDA;
}

}  // namespace net
}  // namespace casl

using namespace casl::net;

struct casl_net {
  int n, device;
  cudaStream_t stream;
  ParamMap m;
  float *w, *mo, *vo, *grad;  // master parameters, Adam moments, flat gradient
  LayerDev L[NL];
  bf16 *x0;                   // input planes (16 channels)
  bf16 *a[3], *z[3];          // activations and pre-activations of layers 1-3
  bf16 *dc;                   // output gradient planes (16 channels)
  bf16 *dz[3];                // pre-activation gradients of layers 1-3
  float *fout;                // [NOUT][n][n] network output
  float *stage;               // host<->device staging, [3][n][n]
  int *err;
  float qscale, uscale;
  int adam_t;
};

namespace casl {
namespace net {

static int fill_zero(cudaStream_t st, void *p, size_t bytes) {
  return cudaMemsetAsync(p, 0, bytes, st) == cudaSuccess ? CASL_OK : CASL_ECUDA;
}

// The forward pass on the packed input x0; train keeps the pre-activations.
int forward(casl_net *N, cudaStream_t st, bool train, int *err) {
  const int n = N->n;
  int rc;
  ConvArgs a{};
  a.n = n;
  a.err = err;
  a.in = N->x0; a.wimg = N->L[0].wf; a.bias = N->L[0].bias; a.out = N->a[0];
  a.zout = train ? N->z[0] : nullptr;
  if ((rc = launch_conv<16, HID, FWD_GELU>(a, st))) return rc;
  for (int l = 1; l < 3; l++) {
    a.in = N->a[l - 1]; a.wimg = N->L[l].wf; a.bias = N->L[l].bias; a.out = N->a[l];
    a.zout = train ? N->z[l] : nullptr;
    if ((rc = launch_conv<HID, HID, FWD_GELU>(a, st))) return rc;
  }
  ConvArgs b{};
  b.n = n; b.err = err;
  b.in = N->a[2]; b.wimg = N->L[3].wf; b.bias = N->L[3].bias; b.fout = N->fout; b.cout_real = NOUT;
  return launch_conv<HID, OUTP, FWD_LINEAR>(b, st);
}

// The backward pass after a training forward, from the packed output
// gradient dc (whose bias sum k_pack_grad has already put in L[3].db); the
// other accumulators are cleared here.
int backward(casl_net *N, cudaStream_t st, int *err) {
  const int n = N->n;
  int rc;
  for (int l = 0; l < NL; l++) {
    if ((rc = fill_zero(st, N->L[l].dw, 25ull * cin_p(l) * cout_p(l) * sizeof(float)))) return rc;
    if (l < 3 && (rc = fill_zero(st, N->L[l].db, cout_p(l) * sizeof(float)))) return rc;
  }
  WgradArgs w{};
  w.n = n; w.err = err;
  w.in = N->a[2]; w.dz = N->dc; w.dw = N->L[3].dw;
  if ((rc = launch_wgrad<HID, OUTP>(w, st))) return rc;
  ConvArgs a{};
  a.n = n; a.err = err;
  a.in = N->dc; a.wimg = N->L[3].wb; a.out = N->dz[2]; a.zprev = N->z[2]; a.dbias = N->L[2].db;
  if ((rc = launch_conv<OUTP, HID, BWD_GELU>(a, st))) return rc;
  for (int l = 2; l >= 1; l--) {
    w.in = N->a[l - 1]; w.dz = N->dz[l]; w.dw = N->L[l].dw;
    if ((rc = launch_wgrad<HID, HID>(w, st))) return rc;
    a.in = N->dz[l]; a.wimg = N->L[l].wb; a.out = N->dz[l - 1]; a.zprev = N->z[l - 1];
    a.dbias = N->L[l - 1].db;
    if ((rc = launch_conv<HID, HID, BWD_GELU>(a, st))) return rc;
  }
  w.in = N->x0; w.dz = N->dz[0]; w.dw = N->L[0].dw;
  return launch_wgrad<16, HID>(w, st);
}

static Params params_of(casl_net *N) {
  Params P{};
  P.w = N->w;
  P.m = N->m;
  for (int l = 0; l < NL; l++) P.L[l] = N->L[l];
  return P;
}

int refresh_images(casl_net *N, cudaStream_t st) {
  CASL_K(k_weight_images, 148, 256, 0, st)(params_of(N));
  return cudaPeekAtLastError() == cudaSuccess ? CASL_OK : CASL_ECUDA;
}

int adam_step(casl_net *N, cudaStream_t st, float lr) {
  N->adam_t++;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.0f - powf(b1, (float)N->adam_t), c2 = 1.0f - powf(b2, (float)N->adam_t);
  CASL_K(k_adam, 148, 256, 0, st)(params_of(N), N->w, N->mo, N->vo, lr, b1, b2, 1e-8f, c1, c2);
  if (cudaPeekAtLastError() != cudaSuccess) return CASL_ECUDA;
  return refresh_images(N, st);
}

static int read_err(casl_net *N, cudaStream_t st) {
  int e = 0;
  if (cudaMemcpyAsync(&e, N->err, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess)
    return CASL_ECUDA;
  if (cudaStreamSynchronize(st) != cudaSuccess) return CASL_ECUDA;
  if (e) {
    int z = 0;
    cudaMemcpy(N->err, &z, sizeof(int), cudaMemcpyHostToDevice);
  }
  return e;
}

}  // namespace net
}  // namespace casl

// ---------------------------------------------------------------------------
// The closure inside the solver
// ---------------------------------------------------------------------------
namespace casl {

struct ClosureState {
  casl_net *net;            // the attached network (not owned); nullptr = none
  casl_handle *judge;       // fine-grid judge for the periodic check (not owned, nullable)
  int check_every;          // steps between checks (0 = never)
  double budget;            // relative node-velocity error the correction may not exceed
  int active;               // the correction is applied inside the step
  long long steps, checks, fallbacks;
  double last_plain, last_net;
  double *uJ, *vJ, *uP, *vP, *uC, *vC;  // node arrays (capacity cap)
  double *du, *dv;          // the correction at the nodes inside a step (capacity cap)
  long long cap;
  float *dcf;               // [NOUT][n][n] output gradient of the node loss
  int *feat;                // [NSUBF][n][n] sub-cell levels, written by con2grid
  double *acc;              // [4] sums of the node errors
};

namespace net {

// The network's input from the inversion of a stage: the contour PV on the
// coarse grid (the integer cells of con2grid with its mean removed, as the
// transform's load forms it), u and v, and the sub-cell levels F that the
// same con2grid wrote, as qjump (L - C/256): the fine level's deviation from
// the cell's weighted mean (the 7 x 7 weights sum to 256); all divided by
// the scales.
template <class T>
__global__ void k_features(const int *__restrict__ C, const int *__restrict__ F,
                           const Scalars *__restrict__ s, const T *__restrict__ uu,
                           const T *__restrict__ vv, float iq, float iu, bf16 *__restrict__ x0,
                           int n, int contex) {
  CASL_PDL_ENTRY();
  const long long nn = (long long)n * n;
  const double inv = 1.0 / (256.0 * (double)n * (double)n);
  const long long S = s->csum;
  const double qj = s->qjump;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nn;
       t += (long long)gridDim.x * blockDim.x) {
    const double q = contex ? qj * ((double)((long long)C[t] * nn - S) * inv) : 0.0;
    float v[16];
    v[0] = (float)q * iq;
    v[1] = (float)uu[t] * iu;
    v[2] = (float)vv[t] * iu;
    const double cm = contex ? (double)C[t] * (1.0 / 256.0) : 0.0;
#pragma unroll
    for (int k = 0; k < NSUBF; k++)
      v[3 + k] = contex && F ? (float)(qj * ((double)F[k * nn + t] - cm)) * iq : 0.0f;
#pragma unroll
    for (int c = NIN; c < 16; c++) v[c] = 0.0f;
    store_px<16>(x0, n, (int)(t / n), (int)(t % n), v);
  }
}

// Corners and weights of the bilinear interpolation of the correction at
// node (x, y) on the SUB-times finer grid, as offsets into one component's
// SUB^2 channels: point (I, J) of the fine grid is sub-cell (I % SUB,
// J % SUB) of coarse cell (I / SUB, J / SUB).  Indices are clamped so that
// no input reads outside the output (valid nodes never need the clamp).
__device__ __forceinline__ void sub_corners(double x, double y, const Consts &c, long long *k,
                                            double *w) {
  const int mx = SUB * c.nx, my = SUB * c.ny;
  const double xx = ((double)SUB * c.glxi) * (x - c.xmin);
  const double yy = ((double)SUB * c.glyi) * (y - c.ymin);
  int i0 = f_int(xx), j0 = f_int(yy);
  const double px = xx - (double)i0, py = yy - (double)j0;
  i0 = i0 < 0 ? 0 : (i0 > mx - 1 ? mx - 1 : i0);
  j0 = j0 < 0 ? 0 : (j0 > my - 1 ? my - 1 : j0);
  const int i1 = i0 + 1 == mx ? 0 : i0 + 1, j1 = j0 + 1 == my ? 0 : j0 + 1;
  const long long nn = (long long)c.nx * c.ny;
  auto at = [&](int I, int J) -> long long {
    return (long long)((I % SUB) * SUB + (J % SUB)) * nn + (long long)(I / SUB) * c.ny + (J / SUB);
  };
  k[0] = at(i0, j0); w[0] = (1.0 - px) * (1.0 - py);
  k[1] = at(i1, j0); w[1] = px * (1.0 - py);
  k[2] = at(i0, j1); w[2] = (1.0 - px) * py;
  k[3] = at(i1, j1); w[3] = px * py;
}

// The correction at the nodes, us * (bilinear interpolation of y on the
// fine grid), added to the plain node velocities (up, vp) when they are
// given.
__global__ void k_corr_nodes(const double *__restrict__ xq, const double *__restrict__ yq,
                             int npt, const float *__restrict__ y, float us, Consts c,
                             const double *__restrict__ up, const double *__restrict__ vp,
                             double *__restrict__ uo, double *__restrict__ vo) {
  CASL_PDL_ENTRY();
  const long long cv = (long long)SUB * SUB * c.nx * c.ny;  // the v channels
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npt; i += gridDim.x * blockDim.x) {
    long long k[4];
    double w[4];
    sub_corners(xq[i], yq[i], c, k, w);
    double du = 0.0, dv = 0.0;
#pragma unroll
    for (int j = 0; j < 4; j++) {
      du += w[j] * (double)y[k[j]];
      dv += w[j] * (double)y[cv + k[j]];
    }
    uo[i] = (up ? up[i] : 0.0) + (double)us * du;
    vo[i] = (vp ? vp[i] : 0.0) + (double)us * dv;
  }
}

// Node errors against the judge: acc[0] += |corrected - judge|^2,
// acc[1] += |plain - judge|^2, acc[2] += |judge|^2.  With g non-null, the
// gradient of the loss sum |corrected - judge|^2 / (npt us^2) with respect
// to the network output is scattered into g ([NOUT][n][n]) with the fine
// grid's bilinear weights.
__global__ void k_node_loss(const double *__restrict__ xq, const double *__restrict__ yq, int npt,
                            const double *__restrict__ uC, const double *__restrict__ vC,
                            const double *__restrict__ uP, const double *__restrict__ vP,
                            const double *__restrict__ uJ, const double *__restrict__ vJ,
                            Consts c, float us, float *__restrict__ g, double *__restrict__ acc) {
  CASL_PDL_ENTRY();
  double s0 = 0.0, s1 = 0.0, s2 = 0.0;
  const long long cv = (long long)SUB * SUB * c.nx * c.ny;  // the v channels
  const double gs = 2.0 / ((double)npt * (double)us);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npt; i += gridDim.x * blockDim.x) {
    const double ru = uC[i] - uJ[i], rv = vC[i] - vJ[i];
    const double pu = uP[i] - uJ[i], pv = vP[i] - vJ[i];
    s0 += ru * ru + rv * rv;
    s1 += pu * pu + pv * pv;
    s2 += uJ[i] * uJ[i] + vJ[i] * vJ[i];
    if (g) {
      long long k[4];
      double w[4];
      sub_corners(xq[i], yq[i], c, k, w);
#pragma unroll
      for (int j = 0; j < 4; j++) {
        atomicAdd(&g[k[j]], (float)(gs * ru * w[j]));
        atomicAdd(&g[cv + k[j]], (float)(gs * rv * w[j]));
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    s0 += __shfl_xor_sync(0xffffffffu, s0, o);
    s1 += __shfl_xor_sync(0xffffffffu, s1, o);
    s2 += __shfl_xor_sync(0xffffffffu, s2, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&acc[0], s0);
    atomicAdd(&acc[1], s1);
    atomicAdd(&acc[2], s2);
  }
}

}  // namespace net

static int cs_grow(ClosureState *cs, long long npt) {
  if (npt <= cs->cap) return CASL_OK;
  double **arrs[] = {&cs->uJ, &cs->vJ, &cs->uP, &cs->vP, &cs->uC, &cs->vC, &cs->du, &cs->dv};
  for (auto a : arrs) {
    cudaFree(*a);
    *a = nullptr;
  }
  const long long cap = npt + npt / 2 + 1024;
  for (auto a : arrs)
    if (cudaMalloc(a, (size_t)cap * sizeof(double)) != cudaSuccess) {
      cs->cap = 0;
      return CASL_ENOMEM;
    }
  cs->cap = cap;
  return CASL_OK;
}

static ClosureState *cs_get(casl_handle *h, int *rc) {
  *rc = CASL_OK;
  if (h->closure) return h->closure;
  ClosureState *cs = (ClosureState *)calloc(1, sizeof(ClosureState));
  if (!cs) {
    *rc = CASL_ENOMEM;
    return nullptr;
  }
  const size_t nn = (size_t)h->n * h->n;
  bool ok = cudaMalloc(&cs->dcf, NOUT * nn * 4) == cudaSuccess && cudaMalloc(&cs->acc, 64) == cudaSuccess &&
            cudaMalloc(&cs->feat, NSUBF * nn * 4) == cudaSuccess &&
            cudaMemset(cs->feat, 0, NSUBF * nn * 4) == cudaSuccess;
  if (!ok) {
    cudaFree(cs->dcf); cudaFree(cs->acc); cudaFree(cs->feat);
    free(cs);
    *rc = CASL_ENOMEM;
    return nullptr;
  }
  h->closure = cs;
  // con2grid writes the network's sub-cell input from now on
  if (h->M == 1) h->c2g_feat = cs->feat;
  return cs;
}

void closure_release(casl_handle *h) {
  ClosureState *cs = h->closure;
  if (!cs) return;
  void *ps[] = {cs->dcf, cs->acc, cs->uJ, cs->vJ, cs->uP, cs->vP, cs->uC, cs->vC, cs->du, cs->dv,
                cs->feat};
  for (void *p : ps) cudaFree(p);
  free(cs);
  h->closure = nullptr;
  h->c2g_feat = nullptr;
}

static inline int gsz(long long work) {
  long long g = (work + 255) / 256;
  return (int)(g < 1 ? 1 : (g > 148 * 16 ? 148 * 16 : g));
}

// Network input and forward (train keeps the pre-activations) from h's
// latest inversion (FP64 fields, or FP32 ones in the FP32-inversion mode),
// on h's stream: the correction is left in N->fout.
template <class T>
static int net_run_t(casl_handle *h, casl_net *N, const T *uu, const T *vv, bool train) {
  const long long nn = (long long)h->n * h->n;
  cudaStream_t st = h->stream;
  CASL_K(net::k_features<T>, gsz(nn), 256, 0, st)(h->coarseC, h->c2g_feat, h->scal, uu, vv,
                                                   1.0f / N->qscale, 1.0f / N->uscale, N->x0,
                                                   h->n, h->nptq > 0 ? 1 : 0);
  return net::forward(N, st, train, &h->scal->error);
}

// The correction at the nodes for a stage's node update: the network on
// the stage's fields, interpolated to the nodes' current positions.
template <class T>
static int closure_stage_t(casl_handle *h, const T *uu, const T *vv, const double **du,
                           const double **dv) {
  ClosureState *cs = h->closure;
  if (!cs || !cs->net || !cs->active || h->nptq == 0) return CASL_OK;
  int rc = cs_grow(cs, h->nptq);
  if (rc) return rc;
  if ((rc = net_run_t<T>(h, cs->net, uu, vv, false))) return rc;
  CASL_K(net::k_corr_nodes, gsz(h->nptq), 256, 0, h->stream)(h->xq, h->yq, h->nptq,
                                                             cs->net->fout, cs->net->uscale, h->c,
                                                             nullptr, nullptr, cs->du, cs->dv);
  *du = cs->du;
  *dv = cs->dv;
  return cudaPeekAtLastError() == cudaSuccess ? CASL_OK : CASL_ECUDA;
}
int closure_stage(casl_handle *h, const double **du, const double **dv) {
  return closure_stage_t<double>(h, h->uu, h->vv, du, dv);
}
int closure_stage32(casl_handle *h, const float *u, const float *v, const double **du,
                    const double **dv) {
  return closure_stage_t<float>(h, u, v, du, dv);
}

// Judge, network and node errors at h's current state: out[0] the plain
// relative error, out[1] the corrected one, out[2] the loss.  With train, the
// loss gradient is back-propagated and one Adam step taken.
static int evaluate(casl_handle *h, casl_net *N, casl_handle *hf, bool train, float lr,
                    double out[3]) {
  int rc;
  ClosureState *cs = cs_get(h, &rc);
  if (!cs) return rc;
  if ((rc = sync_counts(h))) return rc;
  const int npt = h->nptq;
  if (npt == 0) {
    out[0] = out[1] = out[2] = 0.0;
    return CASL_OK;
  }
  if ((rc = cs_grow(cs, npt))) return rc;
  Trace tr;
  tr.begin(h->stream, "evaluate");
  if ((rc = judge_velocity(h, hf, cs->uJ, cs->vJ, cs->uP, cs->vP))) return rc;
  tr.point("judge");
  if ((rc = net_run_t<double>(h, N, h->uu, h->vv, train))) return rc;
  tr.point("network");
  cudaStream_t st = h->stream;
  CASL_K(net::k_corr_nodes, gsz(npt), 256, 0, st)(h->xq, h->yq, npt, N->fout, N->uscale, h->c,
                                                   cs->uP, cs->vP, cs->uC, cs->vC);
  const long long nn = (long long)h->n * h->n;
  if (cudaMemsetAsync(cs->acc, 0, 64, st) != cudaSuccess) return CASL_ECUDA;
  if (train && cudaMemsetAsync(cs->dcf, 0, NOUT * nn * 4, st) != cudaSuccess) return CASL_ECUDA;
  CASL_K(net::k_node_loss, gsz(npt), 256, 0, st)(h->xq, h->yq, npt, cs->uC, cs->vC, cs->uP,
                                                  cs->vP, cs->uJ, cs->vJ, h->c, N->uscale,
                                                  train ? cs->dcf : nullptr, cs->acc);
  if (train) {
    if (cudaMemsetAsync(N->L[3].db, 0, cout_p(3) * 4, st) != cudaSuccess) return CASL_ECUDA;
    CASL_K(net::k_pack_grad<OUTP>, 148 * 4, 256, 0, st)(cs->dcf, N->dc, h->n, NOUT, N->L[3].db);
    if ((rc = net::backward(N, st, &h->scal->error))) return rc;
    if ((rc = net::adam_step(N, st, lr))) return rc;
  }
  tr.point(train ? "loss+backward+adam" : "loss");
  tr.flush("evaluate");
  double a[3];
  if (cudaMemcpyAsync(a, cs->acc, 3 * sizeof(double), cudaMemcpyDeviceToHost, st) != cudaSuccess)
    return CASL_ECUDA;
  if ((rc = sync_counts(h))) return rc;
  out[0] = a[2] > 0.0 ? sqrt(a[1] / a[2]) : 0.0;
  out[1] = a[2] > 0.0 ? sqrt(a[0] / a[2]) : 0.0;
  out[2] = a[0] / ((double)npt * (double)N->uscale * (double)N->uscale);
  return check_launch(h);
}

static int run_check(casl_handle *h, ClosureState *cs) {
  double e[3];
  int rc = evaluate(h, cs->net, cs->judge, false, 0.0f, e);
  if (rc) return rc;
  cs->checks++;
  cs->last_plain = e[0];
  cs->last_net = e[1];
  // the two error sums are accumulated by atomics in different orders, so
  // equal errors can differ in the last bits
  const int ok = e[1] <= cs->budget && e[1] <= e[0] * (1.0 + 1e-9);
  if (!ok && cs->active) cs->fallbacks++;
  cs->active = ok;
  return CASL_OK;
}

int closure_step_check(casl_handle *h) {
  ClosureState *cs = h->closure;
  if (!cs || !cs->net) return CASL_OK;
  const long long k = cs->steps++;
  if (!cs->judge || cs->check_every <= 0 || k % cs->check_every) return CASL_OK;
  return run_check(h, cs);
}

}  // namespace casl

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

int casl_net_param_count(void) { return param_map().total; }

void casl_net_destroy(casl_net *N) {
  if (!N) return;
  cudaSetDevice(N->device);
  cudaStreamSynchronize(N->stream);
  void *ps[] = {N->w, N->mo, N->vo, N->grad, N->x0, N->dc, N->fout, N->stage, N->err};
  for (void *p : ps) cudaFree(p);
  for (int i = 0; i < 3; i++) {
    cudaFree(N->a[i]);
    cudaFree(N->z[i]);
    cudaFree(N->dz[i]);
  }
  for (int l = 0; l < NL; l++) {
    cudaFree(N->L[l].wf);
    cudaFree(N->L[l].wb);
    cudaFree(N->L[l].bias);
    cudaFree(N->L[l].dw);
    cudaFree(N->L[l].db);
  }
  cudaStreamDestroy(N->stream);
  free(N);
}

int casl_net_create(int n, int device, casl_net **out) {
  if (!out || n < 128 || n > 2048 || n % SEG || n % RF || n % RW) return CASL_EINVAL;
  *out = nullptr;
  if (cudaSetDevice(device) != cudaSuccess) return CASL_ECUDA;
  casl_net *N = (casl_net *)calloc(1, sizeof(casl_net));
  if (!N) return CASL_ENOMEM;
  N->n = n;
  N->device = device;
  N->m = param_map();
  N->qscale = N->uscale = 1.0f;
  if (cudaStreamCreateWithFlags(&N->stream, cudaStreamNonBlocking) != cudaSuccess) {
    free(N);
    return CASL_ECUDA;
  }
  bool ok = true;
  auto A = [&](void **p, size_t bytes) {
    if (cudaMalloc(p, bytes) != cudaSuccess) ok = false;
    else cudaMemset(*p, 0, bytes);
  };
  const size_t P = N->m.total;
  A((void **)&N->w, P * 4); A((void **)&N->mo, P * 4); A((void **)&N->vo, P * 4);
  A((void **)&N->grad, P * 4);
  A((void **)&N->x0, act_elems(n, 16) * 2);
  A((void **)&N->dc, act_elems(n, OUTP) * 2);
  for (int i = 0; i < 3; i++) {
    A((void **)&N->a[i], act_elems(n, HID) * 2);
    A((void **)&N->z[i], act_elems(n, HID) * 2);
    A((void **)&N->dz[i], act_elems(n, HID) * 2);
  }
  A((void **)&N->fout, (size_t)NOUT * n * n * 4);
  A((void **)&N->stage, (size_t)(NOUT > NIN ? NOUT : NIN) * n * n * 4);
  A((void **)&N->err, 64);
  for (int l = 0; l < NL; l++) {
    const size_t img = 25ull * cin_p(l) * cout_p(l);
    A((void **)&N->L[l].wf, img * 2);
    A((void **)&N->L[l].wb, img * 2);
    A((void **)&N->L[l].bias, cout_p(l) * 4);
    A((void **)&N->L[l].dw, img * 4);
    A((void **)&N->L[l].db, cout_p(l) * 4);
  }
  if (!ok || cudaDeviceSynchronize() != cudaSuccess) {
    casl_net_destroy(N);
    return CASL_ENOMEM;
  }
  *out = N;
  return CASL_OK;
}

int casl_net_set_params(casl_net *N, const float *params, float qscale, float uscale) {
  if (!N || !params || !(qscale > 0.0f) || !(uscale > 0.0f)) return CASL_EINVAL;
  cudaSetDevice(N->device);
  if (cudaMemcpyAsync(N->w, params, N->m.total * 4, cudaMemcpyHostToDevice, N->stream) !=
      cudaSuccess)
    return CASL_ECUDA;
  cudaMemsetAsync(N->mo, 0, N->m.total * 4, N->stream);
  cudaMemsetAsync(N->vo, 0, N->m.total * 4, N->stream);
  N->adam_t = 0;
  N->qscale = qscale;
  N->uscale = uscale;
  int rc = refresh_images(N, N->stream);
  if (rc) return rc;
  return cudaStreamSynchronize(N->stream) == cudaSuccess ? CASL_OK : CASL_ECUDA;
}

int casl_net_get_params(casl_net *N, float *params, float *qscale, float *uscale) {
  if (!N) return CASL_EINVAL;
  cudaSetDevice(N->device);
  if (params && cudaMemcpyAsync(params, N->w, N->m.total * 4, cudaMemcpyDeviceToHost,
                                N->stream) != cudaSuccess)
    return CASL_ECUDA;
  if (qscale) *qscale = N->qscale;
  if (uscale) *uscale = N->uscale;
  return cudaStreamSynchronize(N->stream) == cudaSuccess ? CASL_OK : CASL_ECUDA;
}

int casl_net_forward(casl_net *N, const float *x, float *y) {
  if (!N || !x || !y) return CASL_EINVAL;
  cudaSetDevice(N->device);
  const int n = N->n;
  const size_t nn = (size_t)n * n;
  cudaStream_t st = N->stream;
  if (cudaMemcpyAsync(N->stage, x, NIN * nn * 4, cudaMemcpyHostToDevice, st) != cudaSuccess)
    return CASL_ECUDA;
  CASL_K(k_pack_input, 148 * 4, 256, 0, st)(N->stage, N->x0, n, NIN);
  int rc = forward(N, st, true, N->err);
  if (rc) return rc;
  if (cudaMemcpyAsync(y, N->fout, NOUT * nn * 4, cudaMemcpyDeviceToHost, st) != cudaSuccess)
    return CASL_ECUDA;
  return read_err(N, st);
}

int casl_net_backward(casl_net *N, const float *dy, float *grad) {
  if (!N || !dy) return CASL_EINVAL;
  cudaSetDevice(N->device);
  const int n = N->n;
  const size_t nn = (size_t)n * n;
  cudaStream_t st = N->stream;
  if (cudaMemcpyAsync(N->stage, dy, NOUT * nn * 4, cudaMemcpyHostToDevice, st) != cudaSuccess)
    return CASL_ECUDA;
  if (cudaMemsetAsync(N->L[3].db, 0, cout_p(3) * 4, st) != cudaSuccess) return CASL_ECUDA;
  CASL_K(k_pack_grad<OUTP>, 148 * 4, 256, 0, st)(N->stage, N->dc, n, NOUT, N->L[3].db);
  int rc = backward(N, st, N->err);
  if (rc) return rc;
  if (grad) {
    CASL_K(k_gather_grad, 148, 256, 0, st)(params_of(N), N->grad);
    if (cudaMemcpyAsync(grad, N->grad, N->m.total * 4, cudaMemcpyDeviceToHost, st) !=
        cudaSuccess)
      return CASL_ECUDA;
  }
  return read_err(N, st);
}

int casl_net_adam(casl_net *N, float lr) {
  if (!N || !(lr > 0.0f)) return CASL_EINVAL;
  cudaSetDevice(N->device);
  int rc = adam_step(N, N->stream, lr);
  if (rc) return rc;
  return read_err(N, N->stream);
}

}  // extern "C"

extern "C" {

int casl_closure_attach(casl_handle *h, casl_net *net, casl_handle *judge, int check_every,
                        double budget) {
  if (!h) return CASL_EINVAL;
  if (!net) {
    if (h->closure) {
      h->closure->net = nullptr;
      h->closure->active = 0;
    }
    return CASL_OK;
  }
  if (net->n != h->n || net->device != h->device || check_every < 0 || !(budget > 0.0))
    return CASL_EINVAL;
  if (h->M > 1) return CASL_EUNSUPPORTED;  // one simulation
  if (judge && (judge->device != h->device || judge->n % h->n)) return CASL_EINVAL;
  cudaSetDevice(h->device);
  int rc;
  casl::ClosureState *cs = casl::cs_get(h, &rc);
  if (!cs) return rc;
  cs->net = net;
  cs->judge = judge;
  cs->check_every = check_every;
  cs->budget = budget;
  cs->active = 1;
  cs->steps = cs->checks = cs->fallbacks = 0;
  cs->last_plain = cs->last_net = 0.0;
  return CASL_OK;
}

int casl_closure_status(casl_handle *h, int *active, double *err_plain, double *err_net,
                        long long *checks, long long *fallbacks) {
  if (!h) return CASL_EINVAL;
  casl::ClosureState *cs = h->closure;
  const bool on = cs && cs->net;
  if (active) *active = on ? cs->active : 0;
  if (err_plain) *err_plain = on ? cs->last_plain : 0.0;
  if (err_net) *err_net = on ? cs->last_net : 0.0;
  if (checks) *checks = on ? cs->checks : 0;
  if (fallbacks) *fallbacks = on ? cs->fallbacks : 0;
  return CASL_OK;
}

int casl_closure_check(casl_handle *h, double *err_plain, double *err_net) {
  if (!h || !h->closure || !h->closure->net || !h->closure->judge) return CASL_EINVAL;
  cudaSetDevice(h->device);
  int rc = casl::run_check(h, h->closure);
  if (rc) return rc;
  if (err_plain) *err_plain = h->closure->last_plain;
  if (err_net) *err_net = h->closure->last_net;
  return CASL_OK;
}

int casl_closure_train(casl_handle *h, casl_net *net, casl_handle *judge, float lr,
                       double out[3]) {
  if (!h || !net || !judge || !out || !(lr > 0.0f) || net->n != h->n) return CASL_EINVAL;
  if (net->device != h->device || judge->device != h->device) return CASL_EINVAL;
  cudaSetDevice(h->device);
  return casl::evaluate(h, net, judge, true, lr, out);
}

int casl_closure_evaluate(casl_handle *h, casl_net *net, casl_handle *judge, double out[3]) {
  if (!h || !net || !judge || !out || net->n != h->n) return CASL_EINVAL;
  if (net->device != h->device || judge->device != h->device) return CASL_EINVAL;
  cudaSetDevice(h->device);
  return casl::evaluate(h, net, judge, false, 0.0f, out);
}

int casl_closure_judge(casl_handle *h, casl_handle *judge, double *uJ, double *vJ, double *uP,
                       double *vP) {
  if (!h || !judge || !uJ || !vJ) return CASL_EINVAL;
  if (judge->device != h->device) return CASL_EINVAL;
  cudaSetDevice(h->device);
  int rc;
  casl::ClosureState *cs = casl::cs_get(h, &rc);
  if (!cs) return rc;
  if ((rc = casl::sync_counts(h))) return rc;
  const int npt = h->nptq;
  if (npt == 0) return CASL_OK;
  if ((rc = casl::cs_grow(cs, npt))) return rc;
  if ((rc = casl::judge_velocity(h, judge, cs->uJ, cs->vJ, cs->uP, cs->vP))) return rc;
  cudaStream_t st = h->stream;
  const size_t b = (size_t)npt * sizeof(double);
  if (cudaMemcpyAsync(uJ, cs->uJ, b, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaMemcpyAsync(vJ, cs->vJ, b, cudaMemcpyDeviceToHost, st) != cudaSuccess)
    return CASL_ECUDA;
  if (uP && cudaMemcpyAsync(uP, cs->uP, b, cudaMemcpyDeviceToHost, st) != cudaSuccess)
    return CASL_ECUDA;
  if (vP && cudaMemcpyAsync(vP, cs->vP, b, cudaMemcpyDeviceToHost, st) != cudaSuccess)
    return CASL_ECUDA;
  return casl::sync_counts(h);
}

// The network's correction at h's nodes from h's latest inversion.
int casl_closure_correction(casl_handle *h, casl_net *net, double *du, double *dv) {
  if (!h || !net || !du || !dv || net->n != h->n) return CASL_EINVAL;
  if (net->device != h->device) return CASL_EINVAL;
  cudaSetDevice(h->device);
  int rc;
  casl::ClosureState *cs = casl::cs_get(h, &rc);
  if (!cs) return rc;
  if ((rc = casl::sync_counts(h))) return rc;
  const int npt = h->nptq;
  if (npt == 0) return CASL_OK;
  if ((rc = casl::cs_grow(cs, npt))) return rc;
  if ((rc = casl::inversion_dev(h, false))) return rc;  // con2grid writes the sub-cell levels
  if ((rc = casl::net_run_t<double>(h, net, h->uu, h->vv, false))) return rc;
  cudaStream_t st = h->stream;
  CASL_K(casl::net::k_corr_nodes, casl::gsz(npt), 256, 0, st)(h->xq, h->yq, npt, net->fout,
                                                             net->uscale, h->c, nullptr, nullptr,
                                                             cs->du, cs->dv);
  const size_t b = (size_t)npt * sizeof(double);
  if (cudaMemcpyAsync(du, cs->du, b, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaMemcpyAsync(dv, cs->dv, b, cudaMemcpyDeviceToHost, st) != cudaSuccess)
    return CASL_ECUDA;
  return casl::sync_counts(h);
}

// The network input of an inversion of h's current state (run here, so that
// con2grid writes the sub-cell levels), (NIN, n, n) float32, already divided
// by net's scales.
int casl_closure_features(casl_handle *h, casl_net *net, float *x) {
  if (!h || !net || !x || net->n != h->n) return CASL_EINVAL;
  cudaSetDevice(h->device);
  int rc;
  if (!casl::cs_get(h, &rc)) return rc;
  if ((rc = casl::inversion_dev(h, false))) return rc;
  const long long nn = (long long)h->n * h->n;
  cudaStream_t st = h->stream;
  CASL_K(casl::net::k_features<double>, casl::gsz(nn), 256, 0, st)(
      h->coarseC, h->c2g_feat, h->scal, h->uu, h->vv, 1.0f / net->qscale, 1.0f / net->uscale,
      net->x0, h->n, h->nptq > 0 ? 1 : 0);
  // unpack channels 0..NIN-1 of the padded planes on the host
  std::vector<uint16_t> buf((size_t)act_elems(h->n, 16));
  if (cudaMemcpyAsync(buf.data(), net->x0, buf.size() * 2, cudaMemcpyDeviceToHost, st) !=
      cudaSuccess)
    return CASL_ECUDA;
  if (cudaStreamSynchronize(st) != cudaSuccess) return CASL_ECUDA;
  const int n = h->n;
  for (int c = 0; c < casl::net::NIN; c++)
    for (int r = 0; r < n; r++)
      for (int q = 0; q < n; q++) {
        const uint32_t bits = (uint32_t)buf[act_off(n, 16, r, q, c / 8) + c % 8] << 16;
        float f;
        memcpy(&f, &bits, 4);
        x[((size_t)c * n + r) * n + q] = f;
      }
  return CASL_OK;
}

}  // extern "C"
