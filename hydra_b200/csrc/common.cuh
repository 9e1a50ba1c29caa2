// Shared definitions of the B200 contour-advection library.
//
// Every translation unit is compiled with -fmad=false: the node arithmetic,
// the grid-line crossing tests and the surgery distance tests must round each
// product and sum separately, exactly as the Fortran reference does on x86-64
// (gfortran without -march flags never contracts to FMA), so that integer
// outcomes (crossing cells, box indices, surgery decisions) are reproduced.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace casl {

// Process-wide count of kernel launches issued by this library.
extern unsigned long long g_launches;

// Per-launch timing (casl_kernel_times): when switched on, every launch is
// bracketed by a pair of CUDA events on its stream and tallied by kernel.
bool kt_begin(const char *name, dim3 grid, dim3 block, size_t smem = 0, cudaStream_t st = 0);
bool kt_end();

// Programmatic dependent launch.  Every kernel of the library is launched
// with programmatic stream serialization allowed and starts with
// CASL_PDL_ENTRY(): it waits until the grid before it in the stream has
// completed and its writes are visible (so stream order is kept), then lets
// the grid after it begin launching, which hides that launch behind its own
// execution.  A kernel launched without the attribute passes the wait at
// once.
#define CASL_PDL_ENTRY() \
  asm volatile("griddepcontrol.wait;\n\tgriddepcontrol.launch_dependents;" ::: "memory")

template <class F>
struct Launch {
  F f;
  dim3 grid, block;
  size_t smem;
  cudaStream_t st;
  template <class... A>
  void operator()(A &&...args) const {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, f, static_cast<A &&>(args)...);
  }
};
template <class F>
Launch<F> launch_of(F f, dim3 grid, dim3 block, size_t smem = 0, cudaStream_t st = 0) {
  return Launch<F>{f, grid, block, smem, st};
}

// Clears or fills up to six word arrays in one kernel launch: in-stream like
// cudaMemsetAsync, but a kernel, so the launches around it keep the
// programmatic overlap.  p is 4-byte aligned, words counts 32-bit words.
struct FillJob {
  void *p;
  long long words;
  unsigned int value;
};
int fill_words(cudaStream_t st, const FillJob *jobs, int njobs);

// Every kernel launch goes through CASL_K(kernel, grid, block, smem, stream)(args);
// it counts the launch (and times it while per-launch timing is on).  The
// for-statement form keeps it a single statement that is safe inside an
// unbraced if/else; its increment runs right after the launch.
#define CASL_K(name, ...)                                                            \
  for (bool casl_once_ = ::casl::kt_begin(#name, __VA_ARGS__); casl_once_;         \
       casl_once_ = ::casl::kt_end())                                               \
  ::casl::launch_of(name, __VA_ARGS__)

// Constants of constants.f90 and contours.f90:17-42, computed once on the
// host by the same operations as the reference's PARAMETER expressions.
struct Consts {
  int nx, ny, nxf, nyf, nxu, nyu, nwx, nwy;
  double ellx, elly, pi, twopi, small, small3, oms;
  double hlx, hlxi, xmin, xmax, hly, hlyi, ymin, ymax;
  double kdsq, srwfm, therm, rekman, beta, aspect;
  double glx, glxi, gly, glyi, garea, dsumi;
  double glxf, glxfi, glyf, glyfi, glxu, glxui, glyu, glyui;
  double amu, ell, dm, dm2, d4small, dmsq, dmi, elf, densf;
  int beffect, btropic, heating, friction;
};

// Fortran intrinsics with the reference's semantics.
__host__ __device__ __forceinline__ double f_dint(double x) { return (double)(long long)x; }
__host__ __device__ __forceinline__ int f_int(double x) { return (int)x; }
__host__ __device__ __forceinline__ double f_sign1(double b) { return copysign(1.0, b); }
__host__ __device__ __forceinline__ int f_isign1(int b) { return b >= 0 ? 1 : -1; }

// Periodic wrap of a displacement: xx - ellx*dble(int(xx*hlxi)).
__host__ __device__ __forceinline__ double wrapd(double xx, double ell, double hli) {
  return xx - ell * f_dint(xx * hli);
}
// Node position wrap: oms*(xx - ellx*dble(int(xx*hlxi))) (evolution.f90:219).
__host__ __device__ __forceinline__ double wrapp(double xx, double ell, double hli, double oms) {
  return oms * (xx - ell * f_dint(xx * hli));
}

// Fire-and-forget global additions: the counters are only read by later
// launches, so no value comes back to the thread.
__device__ __forceinline__ void red_add_u64(unsigned long long *p, unsigned long long v) {
  asm volatile("red.relaxed.gpu.global.add.u64 [%0], %1;" ::"l"(__cvta_generic_to_global(p)), "l"(v)
               : "memory");
}
__device__ __forceinline__ void red_add_s32(int *p, int v) {
  asm volatile("red.relaxed.gpu.global.add.s32 [%0], %1;" ::"l"(__cvta_generic_to_global(p)), "r"(v)
               : "memory");
}

// Device-resident scalars of one simulation (variables.f90 and adapt()).
struct Scalars {
  double t, dt, dt2, dt3, dt6, twist;
  double zzrms, zzmax, uumax, dtmax;
  double qjump;
  unsigned long long zz2_bits;   // max of zz^2 as ordered bits (non-negative doubles)
  unsigned long long uu2_bits;   // max of u^2+v^2
  double zz2_sum;                // sum of zz^2 (deterministic two-level reduction)
  long long csum;                // con2grid: sum of coarse integer cells
  int nq, nptq;                  // current counts (device copy)
  int error;                     // sticky device-side error code
  int pad;
};

}  // namespace casl

#define CASL_CUDA_TRY(expr)                               \
  do {                                                    \
    cudaError_t _e = (expr);                              \
    if (_e != cudaSuccess) return ::casl::set_cuda_error(h, _e); \
  } while (0)
