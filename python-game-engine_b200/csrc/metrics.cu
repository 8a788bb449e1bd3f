// Field reductions for the profiling recorder.
//
// The reference's MetricsRecorder copies a captured field into a float64 buffer and, in
// process(), reduces it with numpy over three scopes (src/cfd/profiling/metrics.py:98-133):
// "all", "interior" (the [1:-1, 1:-1] block) and "boundary" (the rest), metrics.py:7-29,
// with the reducers rms, mean, mean_abs, max, max_abs, std (profiling/config.py:270-299).
// Here one launch reduces the field where it lies: every thread folds its cells into two
// float64 accumulators (interior, boundary) holding count, mean and the sum of squared
// deviations (Welford's update; blocks merged with Chan's formula, so std is a two-pass
// quality result), the sum of |x|, max and max |x|; the last block to finish merges the
// per-block partials and writes 18 values: scope (all, interior, boundary) x reducer
// (rms, mean, mean_abs, max, max_abs, std). NaN propagates into max / max_abs as numpy's
// max does; an empty scope gives NaN.

#include "common.cuh"

namespace sg {

namespace {

constexpr int kStatsThreads = 256;
constexpr int kStatsMaxBlocks = 2 * 148;
constexpr int kStatsFields = 6;  // n, mean, m2, sum |x|, max, max |x|

struct Acc {
  double n, mean, m2, sabs, mx, mxa;
};

__device__ __forceinline__ double max_nan(double a, double b) { return (a != a || b != b) ? a + b : fmax(a, b); }

__device__ __forceinline__ Acc acc_empty() { return Acc{0.0, 0.0, 0.0, 0.0, -INFINITY, -INFINITY}; }

__device__ __forceinline__ void acc_push(Acc& a, double x) {
  a.n += 1.0;
  const double d = x - a.mean;
  a.mean += d / a.n;
  a.m2 += d * (x - a.mean);
  a.sabs += fabs(x);
  a.mx = max_nan(a.mx, x);
  a.mxa = max_nan(a.mxa, fabs(x));
}

__device__ __forceinline__ Acc acc_merge(const Acc& a, const Acc& b) {
  if (b.n == 0.0) return a;
  if (a.n == 0.0) return b;
  const double n = a.n + b.n, d = b.mean - a.mean;
  Acc r;
  r.n = n;
  r.mean = a.mean + d * (b.n / n);
  r.m2 = a.m2 + b.m2 + d * d * (a.n * (b.n / n));
  r.sabs = a.sabs + b.sabs;
  r.mx = max_nan(a.mx, b.mx);
  r.mxa = max_nan(a.mxa, b.mxa);
  return r;
}

__device__ __forceinline__ Acc acc_shfl_down(const Acc& a, int o) {
  Acc r;
  r.n = __shfl_down_sync(0xffffffffu, a.n, o);
  r.mean = __shfl_down_sync(0xffffffffu, a.mean, o);
  r.m2 = __shfl_down_sync(0xffffffffu, a.m2, o);
  r.sabs = __shfl_down_sync(0xffffffffu, a.sabs, o);
  r.mx = __shfl_down_sync(0xffffffffu, a.mx, o);
  r.mxa = __shfl_down_sync(0xffffffffu, a.mxa, o);
  return r;
}

// Merge one accumulator per thread over the block; the result is valid in thread 0.
__device__ Acc block_merge(Acc a, Acc* sm) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) a = acc_merge(a, acc_shfl_down(a, o));
  if (lane == 0) sm[warp] = a;
  __syncthreads();
  if (warp == 0) {
    a = lane < (int)(blockDim.x >> 5) ? sm[lane] : acc_empty();
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) a = acc_merge(a, acc_shfl_down(a, o));
  }
  __syncthreads();
  return a;
}

__device__ __forceinline__ void acc_store(double* p, const Acc& a) {
  p[0] = a.n;
  p[1] = a.mean;
  p[2] = a.m2;
  p[3] = a.sabs;
  p[4] = a.mx;
  p[5] = a.mxa;
}

__device__ __forceinline__ Acc acc_load(const volatile double* p) { return Acc{p[0], p[1], p[2], p[3], p[4], p[5]}; }

__device__ __forceinline__ void write_scope(double* out, const Acc& a) {
  if (a.n == 0.0) {
    for (int r = 0; r < 6; ++r) out[r] = NAN;
    return;
  }
  const double var = a.m2 / a.n;
  out[0] = sqrt(var + a.mean * a.mean);  // rms
  out[1] = a.mean;                       // mean
  out[2] = a.sabs / a.n;                 // mean_abs
  out[3] = a.mx;                         // max
  out[4] = a.mxa;                        // max_abs
  out[5] = sqrt(var);                    // std (ddof 0)
}

// Block b folds rows b, b + gridDim.x, ...; partial[b] holds its (interior, boundary)
// accumulators. The last block to arrive merges them all and resets the arrival counter.
template <typename T>
__global__ void __launch_bounds__(kStatsThreads) k_field_stats(int H, int W, const T* __restrict__ a, int64_t ld,
                                                               unsigned int* counter, double* partial, double* out) {
  __shared__ Acc sm[kStatsThreads / 32];
  __shared__ bool last;
  Acc in = acc_empty(), bd = acc_empty();
  for (int j = blockIdx.x; j < H; j += gridDim.x) {
    const T* row = a + (int64_t)j * ld;
    const bool row_in = j >= 1 && j <= H - 2;
    for (int i = threadIdx.x; i < W; i += blockDim.x) {
      const double x = (double)row[i];
      if (row_in && i >= 1 && i <= W - 2)
        acc_push(in, x);
      else
        acc_push(bd, x);
    }
  }
  in = block_merge(in, sm);
  bd = block_merge(bd, sm);
  if (threadIdx.x == 0) {
    acc_store(partial + (int64_t)blockIdx.x * 2 * kStatsFields, in);
    acc_store(partial + (int64_t)blockIdx.x * 2 * kStatsFields + kStatsFields, bd);
    __threadfence();
    last = atomicAdd(counter, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  const volatile double* vp = partial;
  Acc ti = acc_empty(), tb = acc_empty();
  for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) {
    ti = acc_merge(ti, acc_load(vp + (int64_t)b * 2 * kStatsFields));
    tb = acc_merge(tb, acc_load(vp + (int64_t)b * 2 * kStatsFields + kStatsFields));
  }
  ti = block_merge(ti, sm);
  tb = block_merge(tb, sm);
  if (threadIdx.x == 0) {
    write_scope(out + 0, acc_merge(ti, tb));
    write_scope(out + 6, ti);
    write_scope(out + 12, tb);
    *counter = 0u;
  }
}

constexpr int64_t kStatsCounterBytes = 256;

}  // namespace

}  // namespace sg

using namespace sg;

extern "C" {

int64_t sg_field_stats_workspace_bytes(void) {
  return kStatsCounterBytes + (int64_t)kStatsMaxBlocks * 2 * kStatsFields * (int64_t)sizeof(double);
}

int sg_field_stats(int dtype, int64_t H, int64_t W, const void* field, int64_t ld, void* workspace, double* out,
                   void* stream) {
  SG_REQUIRE(H >= 1 && W >= 1 && H <= (1 << 30) && W <= (1 << 30), "bad grid %lld x %lld", (long long)H,
             (long long)W);
  SG_REQUIRE(field && workspace && out, "null pointer");
  SG_REQUIRE(ld >= W, "row stride below row length");
  SG_REQUIRE(((uintptr_t)workspace & 255) == 0, "workspace must be 256-byte aligned");
  unsigned int* counter = (unsigned int*)workspace;
  double* partial = (double*)((char*)workspace + kStatsCounterBytes);
  const int blocks = (int)(H < kStatsMaxBlocks ? H : kStatsMaxBlocks);
  SG_DISPATCH(dtype, {
    SG_LAUNCH(k_field_stats<T><<<blocks, kStatsThreads, 0, as_stream(stream)>>>((int)H, (int)W, (const T*)field, ld,
                                                                               counter, partial, out));
  });
  return check_launch("sg_field_stats");
}

}  // extern "C"

SG_BOUNDS_ACCESSOR(metrics)
