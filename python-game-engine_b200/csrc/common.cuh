// Shared device/host helpers for the smoke_b200 CUDA library (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <string>

#include "smoke_b200.h"

namespace sg {

// ------------------------------------------------------------------ errors
void set_error(const char* fmt, ...);
int fail(int code, const char* fmt, ...);
int check_launch(const char* what);
// Count of kernel launches issued by this library (read with sg_launch_count()).
void note_launch();
unsigned long long launch_count();

// ------------------------------------------------------------------ bounds-check build
// Built with -DSG_BOUNDS_CHECK=1 (lib/libsmoke_b200_bc.so), the index arithmetic of the
// tiled kernels is checked before each access: SG_IN_BOUNDS(cond) records the source line of
// the first failed check in a per-unit device word (sg_bounds_check reads them) and returns
// false, and the caller skips the access. In the normal build the check is `true` and
// compiles away. Nothing traps: a bad index is reported to the host, the context stays usable.
#ifndef SG_BOUNDS_CHECK
#define SG_BOUNDS_CHECK 0
#endif
#if SG_BOUNDS_CHECK
static __device__ unsigned int g_bounds_line;  // one word per translation unit
__device__ __forceinline__ bool in_bounds(bool ok, unsigned line) {
  if (!ok) atomicCAS(&g_bounds_line, 0u, line);
  return ok;
}
#define SG_IN_BOUNDS(cond) (::sg::in_bounds((cond), __LINE__))
// first failed line of this unit (0: none); clear != 0 resets it
#define SG_BOUNDS_ACCESSOR(unit)                                                          \
  extern "C" int sg_bounds_line_##unit(unsigned* line, int clear) {                       \
    if (cudaMemcpyFromSymbol(line, ::sg::g_bounds_line, sizeof(unsigned)) != cudaSuccess) \
      return SG_ERR_CUDA;                                                                 \
    const unsigned zero = 0;                                                              \
    if (clear && cudaMemcpyToSymbol(::sg::g_bounds_line, &zero, sizeof(unsigned)) != cudaSuccess) \
      return SG_ERR_CUDA;                                                                 \
    return SG_OK;                                                                         \
  }
#else
#define SG_IN_BOUNDS(cond) true
#define SG_BOUNDS_ACCESSOR(unit)                                  \
  extern "C" int sg_bounds_line_##unit(unsigned* line, int) {     \
    *line = 0;                                                    \
    return SG_OK;                                                 \
  }
#endif

// Launch a kernel and count it: SG_LAUNCH(k<T><<<grid, block, smem, stream>>>(args));
#define SG_LAUNCH(...)   \
  do {                   \
    __VA_ARGS__;         \
    ::sg::note_launch(); \
  } while (0)

#define SG_REQUIRE(cond, ...)                        \
  do {                                               \
    if (!(cond)) return ::sg::fail(SG_ERR_ARG, __VA_ARGS__); \
  } while (0)

#define SG_CHECK(x)            \
  do {                         \
    int _rc = (x);             \
    if (_rc != SG_OK) return _rc; \
  } while (0)

#define SG_DISPATCH(dtype, ...)                                     \
  do {                                                              \
    if ((dtype) == SG_F32) {                                        \
      using T = float;                                              \
      __VA_ARGS__                                                   \
    } else if ((dtype) == SG_F64) {                                 \
      using T = double;                                             \
      __VA_ARGS__                                                   \
    } else {                                                        \
      return ::sg::fail(SG_ERR_DTYPE, "unsupported dtype code %d", (int)(dtype)); \
    }                                                               \
  } while (0)

// Compile-time mask kind MM (SG_MASK_OPEN / RING / PLANES) for a validated mask_mode.
#define SG_MASK_DISPATCH(mask_mode, ...)                     \
  do {                                                      \
    if ((mask_mode) == SG_MASK_OPEN) {                      \
      constexpr int MM = SG_MASK_OPEN;                      \
      __VA_ARGS__                                           \
    } else if ((mask_mode) == SG_MASK_RING) {               \
      constexpr int MM = SG_MASK_RING;                      \
      __VA_ARGS__                                           \
    } else {                                                \
      constexpr int MM = SG_MASK_PLANES;                    \
      __VA_ARGS__                                           \
    }                                                       \
  } while (0)

// Compile-time solid kind SM (SG_MASK_NONE / RING / PLANES) for a validated solid_mode.
#define SG_SOLID_DISPATCH(solid_mode, ...)                   \
  do {                                                      \
    if ((solid_mode) == SG_MASK_NONE) {                     \
      constexpr int SM = SG_MASK_NONE;                      \
      __VA_ARGS__                                           \
    } else if ((solid_mode) == SG_MASK_RING) {              \
      constexpr int SM = SG_MASK_RING;                      \
      __VA_ARGS__                                           \
    } else {                                                \
      constexpr int SM = SG_MASK_PLANES;                    \
      __VA_ARGS__                                           \
    }                                                       \
  } while (0)

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// ------------------------------------------------------------------ launch shapes
constexpr int kBX = 32;
constexpr int kBY = 8;
inline dim3 grid2d(int64_t cols, int64_t rows) {
  return dim3((unsigned)((cols + kBX - 1) / kBX), (unsigned)((rows + kBY - 1) / kBY));
}
inline dim3 block2d() { return dim3(kBX, kBY); }

// Row-blocked launches: each thread takes kRows cells of one column, kBY rows apart (a
// warp still reads one contiguous row segment per access), so a thread keeps several
// independent loads in flight.
constexpr int kRows = 4;
inline dim3 grid2d_rows(int64_t cols, int64_t rows) {
  return dim3((unsigned)((cols + kBX - 1) / kBX), (unsigned)((rows + kBY * kRows - 1) / (kBY * kRows)));
}
// j of the thread's q-th row in a row-blocked launch
__device__ __forceinline__ int row_of(int q) { return (blockIdx.y * kRows + q) * blockDim.y + threadIdx.y; }

// ------------------------------------------------------------------ masks
// Face/fluid masks of an H x W cell grid, either explicit planes (as the reference
// passes them) or analytic: SG_MASK_OPEN (all interior faces open) or SG_MASK_RING
// (a box whose outermost cells are solid). MODE fixes the kind at compile time (the
// analytic tests then fold into index comparisons); MODE = -1 reads it from `mode`.
template <int MODE>
struct MasksT {
  const uint8_t* fmu;
  int64_t ldu;
  const uint8_t* fmv;
  int64_t ldv;
  const uint8_t* fl;
  int64_t ldf;
  int mode;
  int H, W;

  __device__ __forceinline__ int kind() const { return MODE < 0 ? mode : MODE; }
  __device__ __forceinline__ bool u(int j, int i) const {
    if (kind() == SG_MASK_PLANES) return fmu[(int64_t)j * ldu + i] != 0;
    if (kind() == SG_MASK_OPEN) return i >= 1 && i <= W - 1;
    return j >= 1 && j <= H - 2 && i >= 2 && i <= W - 2;
  }
  __device__ __forceinline__ bool v(int j, int i) const {
    if (kind() == SG_MASK_PLANES) return fmv[(int64_t)j * ldv + i] != 0;
    if (kind() == SG_MASK_OPEN) return j >= 1 && j <= H - 1;
    return i >= 1 && i <= W - 2 && j >= 2 && j <= H - 2;
  }
  // common/simulation.py:108: a cell is fluid when any of its four faces is open.
  __device__ __forceinline__ bool fluid(int j, int i) const {
    if (kind() == SG_MASK_PLANES && fl) return fl[(int64_t)j * ldf + i] != 0;
    return u(j, i) || u(j, i + 1) || v(j, i) || v(j + 1, i);
  }
  template <int M>
  __host__ __device__ MasksT<M> as() const {
    return MasksT<M>{fmu, ldu, fmv, ldv, fl, ldf, mode, H, W};
  }
};
using Masks = MasksT<-1>;

// Solid cell test of boundaries.py:7-39 (plane: value 1; ring: the outermost cells);
// SM fixes the mode at compile time, -1 takes `mode`.
template <int SM>
__device__ __forceinline__ bool solid_at_t(int mode, const uint8_t* s, int64_t ld, int H, int W, int j, int i) {
  const int md = SM < 0 ? mode : SM;
  if (md == SG_MASK_PLANES) return s[(int64_t)j * ld + i] == 1;
  if (md == SG_MASK_RING) return j == 0 || j == H - 1 || i == 0 || i == W - 1;
  return false;
}
__device__ __forceinline__ bool solid_at(int mode, const uint8_t* s, int64_t ld, int H, int W, int j, int i) {
  return solid_at_t<-1>(mode, s, ld, H, W, j, i);
}

inline Masks make_masks(int mode, int64_t H, int64_t W, const uint8_t* fmu, int64_t ldu, const uint8_t* fmv,
                        int64_t ldv, const uint8_t* fl, int64_t ldf) {
  Masks m;
  m.fmu = fmu;
  m.ldu = ldu;
  m.fmv = fmv;
  m.ldv = ldv;
  m.fl = fl;
  m.ldf = ldf;
  m.mode = mode;
  m.H = (int)H;
  m.W = (int)W;
  return m;
}

// ------------------------------------------------------------------ reference arithmetic
// advection.py:6-49. For float fields Numba evaluates (b - a) in float32 and the rest in
// float64 (every expression meets a Python float); the same order is kept here so a
// float32 result is rounded once from the same double value.
__device__ __forceinline__ int64_t clampi(int64_t v, int64_t lo, int64_t hi) {
  return v < lo ? lo : (v > hi ? hi : v);
}

template <typename T>
__device__ __forceinline__ double lerp_ref(T a, T b, double t) {
  T d = b - a;
  return (double)a + (double)d * t;
}

constexpr double kMagicInt = 4503599627370496.0;  // 2^52

// Exact double of 0 <= k < 2^31 without a conversion instruction (the conversion unit is
// the busiest pipe of the advection kernels): the double whose high word is that of 2^52
// and whose low word is k equals 2^52 + k.
__device__ __forceinline__ double idx_double(int k) { return __hiloint2double(0x43300000, k) - kMagicInt; }

// Clamped floor / ceil of x on [0, n] (n = length - 1) as the reference takes them
// (int(math.floor(x)), int(math.ceil(x)), then clamp; advection.py:31-38), f0 = (double)i0.
// The saturating 32-bit conversion cvt.rmi gives, after the clamp, the reference's floor
// index for every double, NaN and +-Inf included (both end at an edge index).
__device__ __forceinline__ void bracket(double x, int n, int& i0, int& i1, double& f0) {
  i0 = min(max(__double2int_rd(x), 0), n);
  f0 = idx_double(i0);
  // the clamped ceiling is the floor index, plus one where x lies above it (NaN, +-Inf and
  // integral x included: those stay at the floor index, as the saturating cvt.rpi would)
  i1 = min(i0 + (x > f0 ? 1 : 0), n);
}

template <typename T>
__device__ __forceinline__ double sample_ref(const T* __restrict__ f, int64_t ld, int64_t rows, int64_t cols,
                                             double x, double y) {
  const int nc = (int)cols - 1, nr = (int)rows - 1;
  int x0, x1, y0, y1;
  double fx, fy;
  bracket(x, nc, x0, x1, fx);
  bracket(y, nr, y0, y1, fy);
  double tx = x - fx;
  double ty = y - fy;
  const T* r0 = f + (int64_t)y0 * ld;
  const T* r1 = f + (int64_t)y1 * ld;
  T c00 = r0[x0], c10 = r0[x1];
  T c01 = r1[x0], c11 = r1[x1];
  double c0 = lerp_ref(c00, c10, tx);
  double c1 = lerp_ref(c01, c11, tx);
  return c0 + (c1 - c0) * ty;
}

// SplitMix64 finaliser (Steele, Lea, Flood 2014); the plume noise hash.
__host__ __device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

__host__ __device__ __forceinline__ double noise(uint64_t seed, int64_t step, int comp, int64_t j, int64_t i,
                                                 double amp) {
  uint64_t h = mix64(seed ^ mix64((uint64_t)step));
  h = mix64(h ^ (((uint64_t)comp << 62) | ((uint64_t)j << 31) | (uint64_t)i));
  double u = (double)(h >> 11) * (1.0 / 9007199254740992.0);
  return amp * (2.0 * u - 1.0);
}

// ------------------------------------------------------------------ reductions
template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Sum of one value per thread over the block; the result is valid in thread 0.
template <typename T>
__device__ __forceinline__ T block_sum(T v) {
  __shared__ T partial[32];
  int lane = (threadIdx.x + threadIdx.y * blockDim.x) & 31;
  int warp = (threadIdx.x + threadIdx.y * blockDim.x) >> 5;
  int nwarps = (blockDim.x * blockDim.y + 31) >> 5;
  v = warp_sum(v);
  if (lane == 0) partial[warp] = v;
  __syncthreads();
  T s = 0;
  if (warp == 0) {
    s = lane < nwarps ? partial[lane] : (T)0;
    s = warp_sum(s);
  }
  __syncthreads();
  return s;
}

}  // namespace sg
