// Red-black SOR on a checkerboard-split layout (red_black_sor_gauss_seidel.py:8-42).
//
// Cell (j, i) of colour c = (i + j) & 1 lives in plane c at row j, column i >> 1 (row pitch
// ldh elements, the same for both planes). In row j colour c sits at i = 2k + s with
// s = (j + c) & 1, so a colour's cells are contiguous: a half sweep streams the plane it
// updates and the other colour's plane, and reads no cell it does not need. Neighbours of
// (j, k) in the other plane: left k - 1 + s, right k + s, down and up k (rows j -+ 1).
//
// Every update evaluates the reference's expression in the reference's order (masked
// neighbour sum in T, l + r + d + up; the rest in double; one rounding to T), as
// k_rbsor_half does on the natural layout, so both layouts give bit-identical iterates.
// Compiled with -fmad=false like the other operator units.
//
// Kernels:
//   k_rbsor_split_half  one colour, in place, one 16-byte cell vector per thread
//   k_rbsor_split_tiles several sweeps per launch: a 32 x 64 tile plus a halo of one cell
//                       per half sweep is staged in shared memory (split planes), swept
//                       there with the valid region shrinking by one cell per half sweep,
//                       and the tile's own cells are written to the other state buffer
//   k_rbsor_split_sumsq / k_sumsq_finalize  deterministic sum of squares of the reference
//                       residual (residual.py:39-40) over the split planes
//   k_mixed_residual, k_add_correction, k_widen, k_narrow  float64 iterative refinement
//                       around float32 sweeps
#include <algorithm>

#include "common.cuh"

namespace sg {

template <typename T>
struct Vec16;
template <>
struct Vec16<float> {
  using type = float4;
  static constexpr int N = 4;
};
template <>
struct Vec16<double> {
  using type = double2;
  static constexpr int N = 2;
};

template <typename T>
__device__ __forceinline__ void vec_to_array(const typename Vec16<T>::type& v, T* a);
template <>
__device__ __forceinline__ void vec_to_array<float>(const float4& v, float* a) {
  a[0] = v.x;
  a[1] = v.y;
  a[2] = v.z;
  a[3] = v.w;
}
template <>
__device__ __forceinline__ void vec_to_array<double>(const double2& v, double* a) {
  a[0] = v.x;
  a[1] = v.y;
}
template <typename T>
__device__ __forceinline__ typename Vec16<T>::type array_to_vec(const T* a);
template <>
__device__ __forceinline__ float4 array_to_vec<float>(const float* a) {
  return make_float4(a[0], a[1], a[2], a[3]);
}
template <>
__device__ __forceinline__ double2 array_to_vec<double>(const double* a) {
  return make_double2(a[0], a[1]);
}

// red_black_sor_gauss_seidel.py:19-25: the SOR value of a cell from its current value c,
// its four (masked, clamped) neighbours and its divergence.
template <typename T>
__device__ __forceinline__ T sor_value(T c, T l, T r, T d, T up, T dv, double alpha, double rb, double omega) {
  T s = l + r;
  s = s + d;
  s = s + up;
  double np_ = ((double)s + alpha * (double)dv) * rb;
  return (T)((1.0 - omega) * (double)c + omega * np_);
}

// ------------------------------------------------------------------ layout conversion
// natural (H x W, stride ld) -> planes (H x ldh each); slots past a row's last cell get 0
template <typename T>
__global__ void k_split_pack(int H, int W, const T* __restrict__ src, int64_t ld, T* __restrict__ p0,
                             T* __restrict__ p1, int64_t ldh) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (j >= H || k >= ldh) return;
  const int s0 = j & 1;  // column offset of colour 0 in row j
  const int i0 = 2 * k + s0, i1 = 2 * k + (1 - s0);
  const T* row = src + (int64_t)j * ld;
  p0[(int64_t)j * ldh + k] = i0 < W ? row[i0] : (T)0;
  p1[(int64_t)j * ldh + k] = i1 < W ? row[i1] : (T)0;
}

template <typename T>
__global__ void k_split_unpack(int H, int W, const T* __restrict__ p0, const T* __restrict__ p1, int64_t ldh,
                               T* __restrict__ dst, int64_t ld) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (j >= H || i >= W) return;
  const T* plane = ((i + j) & 1) ? p1 : p0;
  dst[(int64_t)j * ld + i] = plane[(int64_t)j * ldh + (i >> 1)];
}

// ------------------------------------------------------------------ one colour, streaming
template <typename T, int MM>
__global__ void __launch_bounds__(256) k_rbsor_split_half(int H, int W, T* __restrict__ own,
                                                          const T* __restrict__ oth, const T* __restrict__ dvc,
                                                          int64_t ldh, MasksT<MM> m, double alpha, double rb,
                                                          double omega, int color) {
  constexpr int N = Vec16<T>::N;
  using V = typename Vec16<T>::type;
  const int kv = (blockIdx.x * blockDim.x + threadIdx.x) * N;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int nk = (W + 1) >> 1;
  if (j >= H || kv >= nk) return;
  const int s = (j + color) & 1;
  const int64_t row = (int64_t)j * ldh;
  if (!SG_IN_BOUNDS(kv + N <= ldh && j >= 0)) return;
  T cc[N], dd[N], oo[N], dn[N], up[N];
  vec_to_array<T>(*reinterpret_cast<const V*>(own + row + kv), cc);
  vec_to_array<T>(*reinterpret_cast<const V*>(dvc + row + kv), dd);
  vec_to_array<T>(*reinterpret_cast<const V*>(oth + row + kv), oo);
  if (j > 0) vec_to_array<T>(*reinterpret_cast<const V*>(oth + row - ldh + kv), dn);
  if (j < H - 1) vec_to_array<T>(*reinterpret_cast<const V*>(oth + row + ldh + kv), up);
  // the other colour one slot beyond the vector: k0 - 1 (s = 0) or k0 + N (s = 1)
  T ext = (T)0;
  if (s == 0 && kv > 0) ext = oth[row + kv - 1];
  if (s == 1 && kv + N < nk) ext = oth[row + kv + N];
#pragma unroll
  for (int q = 0; q < N; ++q) {
    const int i = 2 * (kv + q) + s;
    if (i >= W || !m.fluid(j, i)) continue;
    const T c = cc[q];
    const T ol = s == 0 ? (q == 0 ? ext : oo[q - 1]) : oo[q];
    const T orr = s == 0 ? oo[q] : (q == N - 1 ? ext : oo[q + 1]);
    const T l = m.u(j, i) ? (i > 0 ? ol : c) : c;
    const T r = m.u(j, i + 1) ? (i < W - 1 ? orr : c) : c;
    const T d = m.v(j, i) ? (j > 0 ? dn[q] : c) : c;
    const T u = m.v(j + 1, i) ? (j < H - 1 ? up[q] : c) : c;
    cc[q] = sor_value(c, l, r, d, u, dd[q], alpha, rb, omega);
  }
  *reinterpret_cast<V*>(own + row + kv) = array_to_vec<T>(cc);
}

// ------------------------------------------------------------------ several sweeps per launch
constexpr int kTileRows = 32;    // owned rows of a tile
constexpr int kTileCols = 64;    // owned columns (even: tile origins are even, so colours match)
constexpr int kTileThreads = 512;

template <int G>
struct TileShape {
  static constexpr int RR = kTileRows + 2 * G;        // staged rows
  static constexpr int KK = (kTileCols + 2 * G) / 2;  // staged split columns per plane
  static constexpr int KP = KK + 1;                   // shared-memory row pitch
};

template <typename T, int G>
constexpr size_t tile_smem_bytes() {
  return (size_t)4 * TileShape<G>::RR * TileShape<G>::KP * sizeof(T);
}

// Reads state planes (a0, a1) and the divergence planes (d0, d1), runs `half_sweeps`
// (<= G, even) half sweeps on the staged region and writes the tile's own cells to (b0, b1).
// A staged cell next to a region edge that is not the grid's edge lacks a neighbour, so the
// region updated by half sweep h leaves out h + 1 cells along such edges; after
// half_sweeps <= G of them the owned cells (G from those edges) hold exactly the iterates of
// the grid-wide sweeps. Input and output states differ, so no block reads a cell another
// block writes.
template <typename T, int MM, int G>
__global__ void __launch_bounds__(kTileThreads) k_rbsor_split_tiles(int H, int W, const T* __restrict__ a0,
                                                                     const T* __restrict__ a1, T* __restrict__ b0,
                                                                     T* __restrict__ b1, const T* __restrict__ d0,
                                                                     const T* __restrict__ d1, int64_t ldh,
                                                                     MasksT<MM> m, double alpha, double rb,
                                                                     double omega, int half_sweeps) {
  using S = TileShape<G>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* sp = reinterpret_cast<T*>(smem_raw);  // [2][RR][KP] state, then [2][RR][KP] divergence
  T* sd = sp + 2 * S::RR * S::KP;
  const int j0 = blockIdx.y * kTileRows, i0 = blockIdx.x * kTileCols;
  const int R0 = max(j0 - G, 0), R1 = min(j0 + kTileRows + G, H);
  const int C0 = max(i0 - G, 0), C1 = min(i0 + kTileCols + G, W);  // C0 even
  const int kb = C0 >> 1;
  const int nkk = (C1 - C0 + 1) >> 1;  // staged split columns (<= KK)
  const int nrr = R1 - R0;
  const int tid = threadIdx.x;
  for (int e = tid; e < nrr * nkk; e += kTileThreads) {
    const int rr = e / nkk, kk = e - rr * nkk;
    const int64_t g = (int64_t)(R0 + rr) * ldh + kb + kk;
    const int sidx = rr * S::KP + kk;
    if (!SG_IN_BOUNDS(R0 + rr < H && kb + kk < ldh && rr < S::RR && kk < S::KK)) continue;
    sp[sidx] = a0[g];
    sp[S::RR * S::KP + sidx] = a1[g];
    sd[sidx] = d0[g];
    sd[S::RR * S::KP + sidx] = d1[g];
  }
  __syncthreads();
  const int warp = tid >> 5, lane = tid & 31;
  constexpr int kWarps = kTileThreads / 32;
  for (int h = 0; h < half_sweeps; ++h) {
    const int c = h & 1;
    const int rlo = R0 + (R0 > 0 ? h + 1 : 0), rhi = R1 - (R1 < H ? h + 1 : 0);
    const int clo = C0 + (C0 > 0 ? h + 1 : 0), chi = C1 - (C1 < W ? h + 1 : 0);
    T* own = sp + c * S::RR * S::KP;
    const T* oth = sp + (1 - c) * S::RR * S::KP;
    const T* dv = sd + c * S::RR * S::KP;
    for (int j = rlo + warp; j < rhi; j += kWarps) {
      const int s = (j + c) & 1;
      const int rr = j - R0;
      for (int kk = lane; kk < nkk; kk += 32) {
        const int i = C0 + 2 * kk + s;
        if (i < clo || i >= chi || !m.fluid(j, i)) continue;
        const int sidx = rr * S::KP + kk;
        if (!SG_IN_BOUNDS(rr >= 1 - (j == 0) && rr + 1 < S::RR + (j == H - 1) && kk + s <= S::KK &&
                          (i == 0 || kk - 1 + s >= 0)))
          continue;
        const T cv = own[sidx];
        const T l = m.u(j, i) ? (i > 0 ? oth[max(sidx - 1 + s, 0)] : cv) : cv;
        const T r = m.u(j, i + 1) ? (i < W - 1 ? oth[sidx + s] : cv) : cv;
        const T d = m.v(j, i) ? (j > 0 ? oth[sidx - S::KP] : cv) : cv;
        const T u = m.v(j + 1, i) ? (j < H - 1 ? oth[sidx + S::KP] : cv) : cv;
        own[sidx] = sor_value(cv, l, r, d, u, dv[sidx], alpha, rb, omega);
      }
    }
    __syncthreads();
  }
  // the tile's own cells (both colours) to the output state
  const int ohi = min(j0 + kTileRows, H);
  const int ochi = min(i0 + kTileCols, W);
  const int kown = kTileCols / 2;
  for (int e = tid; e < (ohi - j0) * 2 * kown; e += kTileThreads) {
    const int jr = e / (2 * kown);
    const int rem = e - jr * 2 * kown;
    const int c = rem / kown, kq = rem - c * kown;
    const int j = j0 + jr;
    const int k = (i0 >> 1) + kq;
    const int i = 2 * k + ((j + c) & 1);
    if (i >= ochi) continue;
    const int sidx = (j - R0) * S::KP + (k - kb);
    if (!SG_IN_BOUNDS(j < H && k < ldh && k - kb >= 0 && k - kb < S::KK && j - R0 < S::RR)) continue;
    (c ? b1 : b0)[(int64_t)j * ldh + k] = sp[c * S::RR * S::KP + sidx];
  }
}

// ------------------------------------------------------------------ residual norm
// Sum over fluid cells of the squared reference residual r = (nbsum + alpha div) - beta p
// (residual.py:39-40, rounded to T as the natural-layout kernel stores it); with zero_p the
// residual of p = 0, i.e. alpha div on fluid cells. One partial sum per block.
template <typename T, int MM>
__global__ void __launch_bounds__(256) k_rbsor_split_sumsq(int H, int W, const T* __restrict__ p0,
                                                           const T* __restrict__ p1, const T* __restrict__ d0,
                                                           const T* __restrict__ d1, int64_t ldh, MasksT<MM> m,
                                                           double alpha, double beta, int zero_p,
                                                           double* __restrict__ partials) {
  double sq = 0.0;
  const int64_t total = (int64_t)H * W;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int j = (int)(e / W), i = (int)(e - (int64_t)j * W);
    if (!m.fluid(j, i)) continue;
    const int c = (i + j) & 1;
    const T* own = c ? p1 : p0;
    const T* oth = c ? p0 : p1;
    const int k = i >> 1;
    const int64_t g = (int64_t)j * ldh + k;
    const int s = (j + c) & 1;
    const T cv = zero_p ? (T)0 : own[g];
    T l = cv, r = cv, d = cv, u = cv;
    if (!zero_p) {
      if (m.u(j, i) && i > 0) l = oth[g - 1 + s];
      if (m.u(j, i + 1) && i < W - 1) r = oth[g + s];
      if (m.v(j, i) && j > 0) d = oth[g - ldh];
      if (m.v(j + 1, i) && j < H - 1) u = oth[g + ldh];
    }
    T sum = l + r;
    sum = sum + d;
    sum = sum + u;
    const T dv = (c ? d1 : d0)[g];
    const T res = (T)(((double)sum + alpha * (double)dv) - beta * (double)cv);
    sq += (double)res * (double)res;
  }
  const double b = block_sum(sq);
  if (threadIdx.x == 0) partials[blockIdx.x] = b;
}

__global__ void __launch_bounds__(256) k_sumsq_finalize(const double* __restrict__ partials, int n,
                                                        double* __restrict__ out) {
  double s = 0.0;
  for (int k = threadIdx.x; k < n; k += blockDim.x) s += partials[k];
  s = block_sum(s);
  if (threadIdx.x == 0) out[0] = s;
}

// ------------------------------------------------------------------ mixed precision (FP64 refinement)
// Iterative refinement around float32 sweeps: the pressure is accumulated in float64 (p64,
// natural layout, row pitch W), the residual r = (nbsum(p64) + alpha div) - beta p64 of the
// reference (residual.py:39-40) is formed in float64, and its float32 rounding is the rhs of
// the correction equation that the float32 split-layout sweeps solve from zero (alpha = 1).
__global__ void k_widen(int H, int W, const float* __restrict__ p, int64_t ldp, double* __restrict__ p64) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i < W && j < H) p64[(int64_t)j * W + i] = (double)p[(int64_t)j * ldp + i];
}

__global__ void k_narrow(int H, int W, const double* __restrict__ p64, float* __restrict__ p, int64_t ldp) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i < W && j < H) p[(int64_t)j * ldp + i] = (float)p64[(int64_t)j * W + i];
}

// r64 of every cell (0 off the fluid), its float32 rounding into the split rhs planes
// (r0, r1) when they are given, and one partial sum of r64^2 per block. zero_p: the residual
// of p = 0.
template <int MM>
__global__ void __launch_bounds__(256) k_mixed_residual(int H, int W, const double* __restrict__ p64,
                                                        const float* __restrict__ div, int64_t ldd, MasksT<MM> m,
                                                        double alpha, double beta, int zero_p,
                                                        float* __restrict__ r0, float* __restrict__ r1, int64_t ldh,
                                                        double* __restrict__ partials) {
  double sq = 0.0;
  const int64_t total = (int64_t)H * W;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int j = (int)(e / W), i = (int)(e - (int64_t)j * W);
    double res = 0.0;
    if (m.fluid(j, i)) {
      const double c = zero_p ? 0.0 : p64[e];
      double l = c, r = c, d = c, u = c;
      if (!zero_p) {
        if (m.u(j, i) && i > 0) l = p64[e - 1];
        if (m.u(j, i + 1) && i < W - 1) r = p64[e + 1];
        if (m.v(j, i) && j > 0) d = p64[e - W];
        if (m.v(j + 1, i) && j < H - 1) u = p64[e + W];
      }
      const double s = ((l + r) + d) + u;
      res = (s + alpha * (double)div[(int64_t)j * ldd + i]) - beta * c;
    }
    sq += res * res;
    if (r0) (((i + j) & 1) ? r1 : r0)[(int64_t)j * ldh + (i >> 1)] = (float)res;
  }
  const double b = block_sum(sq);
  if (threadIdx.x == 0) partials[blockIdx.x] = b;
}

// p64 += e (the float32 correction held in the split state planes)
__global__ void k_add_correction(int H, int W, const float* __restrict__ e0, const float* __restrict__ e1, int64_t ldh,
                                 double* __restrict__ p64) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= W || j >= H) return;
  const float* plane = ((i + j) & 1) ? e1 : e0;
  p64[(int64_t)j * W + i] += (double)plane[(int64_t)j * ldh + (i >> 1)];
}

// ------------------------------------------------------------------ host side
constexpr int kSumBlocks = 592;  // 4 x 148 SMs

struct SplitWs {
  int64_t ldh;
  size_t plane;  // bytes of one plane (256-byte multiple)
  char* base;
  void* a[2];
  void* b[2];
  void* d[2];
  double* partials;
  double* result;  // [0] sum of squares of p, [1] of p = 0
};

static int64_t split_pitch(int64_t W) { return ((((W + 1) >> 1) + 31) / 32) * 32; }

static size_t split_bytes(int64_t elem, int64_t H, int64_t W, SplitWs* ws, void* base) {
  const int64_t ldh = split_pitch(W);
  const size_t plane = (size_t)(((H * ldh * elem) + 255) / 256 * 256);
  const size_t total = 6 * plane + (size_t)kSumBlocks * 8 + 256;
  if (ws) {
    char* b = (char*)base;
    ws->ldh = ldh;
    ws->plane = plane;
    ws->base = b;
    for (int c = 0; c < 2; ++c) {
      ws->a[c] = b + c * plane;
      ws->b[c] = b + (2 + c) * plane;
      ws->d[c] = b + (4 + c) * plane;
    }
    ws->partials = (double*)(b + 6 * plane);
    ws->result = (double*)(b + 6 * plane + (size_t)kSumBlocks * 8);
  }
  return total;
}

static size_t mixed_bytes(int64_t H, int64_t W, SplitWs* ws, double** p64, void* base) {
  const size_t split = split_bytes(4, H, W, ws, base);
  const size_t wide = (size_t)((H * W * 8 + 255) / 256 * 256);
  if (p64) *p64 = (double*)((char*)base + split);
  return split + wide;
}

static int split_bind(int dtype, int64_t H, int64_t W, void* workspace, int64_t workspace_bytes, SplitWs* ws) {
  if (dtype != SG_F32 && dtype != SG_F64) return fail(SG_ERR_DTYPE, "unsupported dtype code %d", dtype);
  if (H < 1 || W < 1 || H > (1 << 28) || W > (1 << 28)) return fail(SG_ERR_ARG, "bad grid %lld x %lld", (long long)H, (long long)W);
  if (!workspace || ((uintptr_t)workspace & 255)) return fail(SG_ERR_ARG, "workspace must be non-null and 256-byte aligned");
  const int64_t elem = dtype == SG_F32 ? 4 : 8;
  const size_t need = split_bytes(elem, H, W, nullptr, nullptr);
  if ((size_t)workspace_bytes < need)
    return fail(SG_ERR_ARG, "workspace of %lld bytes below the %zu required", (long long)workspace_bytes, need);
  split_bytes(elem, H, W, ws, workspace);
  return SG_OK;
}

// Variant -1 (automatic): the shared-memory tiles while the state and divergence planes fit
// well inside L2 (their launches are latency-bound there and the tiles do 4 sweeps per
// launch), the streaming half sweeps above that (bandwidth-bound; the tiles' redundant halo
// work then costs more than it saves).
static int resolve_variant(int variant, int64_t H, int64_t W, int64_t elem) {
  if (variant >= 0) return variant;
  return H * W * elem * 2 <= ((int64_t)8 << 20) ? 1 : 0;
}

template <typename T, int MM>
static void launch_half(int H, int W, const SplitWs& w, MasksT<MM> m, double alpha, double rb, double omega, int color,
                        cudaStream_t s) {
  constexpr int N = Vec16<T>::N;
  const int nk = (W + 1) >> 1;
  dim3 block(32, 8);
  dim3 grid((unsigned)((nk + 32 * N - 1) / (32 * N)), (unsigned)((H + 7) / 8));
  SG_LAUNCH(k_rbsor_split_half<T, MM><<<grid, block, 0, s>>>(H, W, (T*)w.a[color], (const T*)w.a[1 - color],
                                                             (const T*)w.d[color], w.ldh, m, alpha, rb, omega, color));
}

constexpr int kTileHalo = 8;  // halo of the tile kernel: up to 4 sweeps per launch

template <typename T, int MM>
static int launch_tiles(int H, int W, const SplitWs& w, bool a_to_b, MasksT<MM> m, double alpha, double rb,
                        double omega, int sweeps, cudaStream_t s) {
  constexpr size_t smem = tile_smem_bytes<T, kTileHalo>();
  // set on every launch: the limit belongs to the function in the current device's context
  cudaError_t e = cudaFuncSetAttribute(k_rbsor_split_tiles<T, MM, kTileHalo>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return fail(SG_ERR_CUDA, "cudaFuncSetAttribute: %s", cudaGetErrorString(e));
  dim3 grid((unsigned)((W + kTileCols - 1) / kTileCols), (unsigned)((H + kTileRows - 1) / kTileRows));
  void* const* src = a_to_b ? w.a : w.b;
  void* const* dst = a_to_b ? w.b : w.a;
  SG_LAUNCH(k_rbsor_split_tiles<T, MM, kTileHalo><<<grid, kTileThreads, smem, s>>>(
      H, W, (const T*)src[0], (const T*)src[1], (T*)dst[0], (T*)dst[1], (const T*)w.d[0], (const T*)w.d[1], w.ldh, m,
      alpha, rb, omega, 2 * sweeps));
  return SG_OK;
}

// `iterations` sweeps on state a (the result ends in a). variant 0: two streaming half-sweep
// launches per sweep; variant 1: tile launches of up to kTileHalo / 2 sweeps each, an even
// number of them (a -> b -> a ...), or streaming launches for a single sweep.
template <typename T, int MM>
static int split_sweeps(int H, int W, const SplitWs& w, MasksT<MM> m, double alpha, double rb, double omega,
                        int64_t iterations, int variant, cudaStream_t s) {
  if (iterations <= 0) return SG_OK;
  if (variant == 0 || iterations == 1) {
    for (int64_t it = 0; it < iterations; ++it)
      for (int color = 0; color < 2; ++color) launch_half<T, MM>(H, W, w, m, alpha, rb, omega, color, s);
    return SG_OK;
  }
  constexpr int per = kTileHalo / 2;
  int64_t launches = (iterations + per - 1) / per;
  if (launches & 1) ++launches;  // iterations >= 2, so every launch still gets >= 1 sweep
  const int64_t base = iterations / launches, extra = iterations % launches;
  for (int64_t q = 0; q < launches; ++q) {
    const int n = (int)(base + (q < extra ? 1 : 0));
    SG_CHECK((launch_tiles<T, MM>(H, W, w, (q & 1) == 0, m, alpha, rb, omega, n, s)));
  }
  return SG_OK;
}

template <typename T, int MM>
static void split_sumsq(int H, int W, const SplitWs& w, MasksT<MM> m, double alpha, double beta, int zero_p,
                        double* out, cudaStream_t s) {
  const int64_t cells = (int64_t)H * W;
  const int blocks = (int)std::min<int64_t>(kSumBlocks, (cells + 255) / 256);
  SG_LAUNCH(k_rbsor_split_sumsq<T, MM><<<blocks, 256, 0, s>>>(H, W, (const T*)w.a[0], (const T*)w.a[1],
                                                              (const T*)w.d[0], (const T*)w.d[1], w.ldh, m, alpha,
                                                              beta, zero_p, w.partials));
  SG_LAUNCH(k_sumsq_finalize<<<1, 256, 0, s>>>(w.partials, blocks, out));
}

static int read_scalar(const double* dptr, double* host, cudaStream_t s) {
  cudaError_t e = cudaMemcpyAsync(host, dptr, sizeof(double), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return fail(SG_ERR_CUDA, "residual read: %s", cudaGetErrorString(e));
  return SG_OK;
}

}  // namespace sg

using namespace sg;

static int split_mask_check(int mode, const void* a, const void* b) {
  if (mode == SG_MASK_PLANES) {
    if (!a || !b) return fail(SG_ERR_ARG, "mask planes required in SG_MASK_PLANES mode");
    return SG_OK;
  }
  if (mode == SG_MASK_OPEN || mode == SG_MASK_RING) return SG_OK;
  return fail(SG_ERR_ARG, "bad mask mode %d", mode);
}

extern "C" {

int64_t sg_rbsor_split_workspace_bytes(int dtype, int64_t H, int64_t W) {
  if ((dtype != SG_F32 && dtype != SG_F64) || H < 1 || W < 1) return -1;
  return (int64_t)split_bytes(dtype == SG_F32 ? 4 : 8, H, W, nullptr, nullptr);
}

int sg_rbsor_split_pack(int dtype, int64_t H, int64_t W, const void* src, int64_t ld_src, int which, void* workspace,
                        int64_t workspace_bytes, void* stream) {
  SplitWs w{};
  SG_CHECK(split_bind(dtype, H, W, workspace, workspace_bytes, &w));
  SG_REQUIRE(src && ld_src >= W, "bad source field");
  SG_REQUIRE(which == 0 || which == 1, "which must be 0 (pressure) or 1 (divergence)");
  void* const* dst = which == 0 ? w.a : w.d;
  dim3 grid((unsigned)((w.ldh + 31) / 32), (unsigned)((H + 7) / 8));
  SG_DISPATCH(dtype, {
    SG_LAUNCH(k_split_pack<T><<<grid, dim3(32, 8), 0, as_stream(stream)>>>((int)H, (int)W, (const T*)src, ld_src,
                                                                         (T*)dst[0], (T*)dst[1], w.ldh));
  });
  return check_launch("sg_rbsor_split_pack");
}

int sg_rbsor_split_unpack(int dtype, int64_t H, int64_t W, const void* workspace, int64_t workspace_bytes, void* dst,
                          int64_t ld_dst, void* stream) {
  SplitWs w{};
  SG_CHECK(split_bind(dtype, H, W, (void*)workspace, workspace_bytes, &w));
  SG_REQUIRE(dst && ld_dst >= W, "bad destination field");
  SG_DISPATCH(dtype, {
    SG_LAUNCH(k_split_unpack<T><<<grid2d(W, H), block2d(), 0, as_stream(stream)>>>((int)H, (int)W, (const T*)w.a[0],
                                                                                 (const T*)w.a[1], w.ldh, (T*)dst,
                                                                                 ld_dst));
  });
  return check_launch("sg_rbsor_split_unpack");
}

int sg_rbsor_split_sweeps(int dtype, int64_t H, int64_t W, void* workspace, int64_t workspace_bytes, int mask_mode,
                          const uint8_t* fmu, int64_t ld_fmu, const uint8_t* fmv, int64_t ld_fmv, double alpha,
                          double reciprocal_beta, double omega, int64_t iterations, int variant, void* stream) {
  SplitWs w{};
  SG_CHECK(split_bind(dtype, H, W, workspace, workspace_bytes, &w));
  SG_REQUIRE(iterations >= 0, "iterations must be >= 0");
  SG_REQUIRE(variant >= -1 && variant <= 1, "variant must be -1 (automatic), 0 (half-sweep launches) or 1 (tiles)");
  SG_CHECK(split_mask_check(mask_mode, fmu, fmv));
  Masks m = make_masks(mask_mode, H, W, fmu, ld_fmu, fmv, ld_fmv, nullptr, 0);
  cudaStream_t s = as_stream(stream);
  SG_DISPATCH(dtype, {
    const int var = resolve_variant(variant, H, W, sizeof(T));
    SG_MASK_DISPATCH(mask_mode, {
      SG_CHECK((split_sweeps<T, MM>((int)H, (int)W, w, m.as<MM>(), alpha, reciprocal_beta, omega, iterations, var,
                                    s)));
    });
  });
  return check_launch("sg_rbsor_split_sweeps");
}

int sg_rbsor_split_sumsq(int dtype, int64_t H, int64_t W, void* workspace, int64_t workspace_bytes, int mask_mode,
                         const uint8_t* fmu, int64_t ld_fmu, const uint8_t* fmv, int64_t ld_fmv, double alpha,
                         double reciprocal_beta, int zero_p, double* out, void* stream) {
  SplitWs w{};
  SG_CHECK(split_bind(dtype, H, W, workspace, workspace_bytes, &w));
  SG_REQUIRE(out, "null output");
  SG_REQUIRE(reciprocal_beta != 0.0, "reciprocal_beta must be non-zero");
  SG_CHECK(split_mask_check(mask_mode, fmu, fmv));
  Masks m = make_masks(mask_mode, H, W, fmu, ld_fmu, fmv, ld_fmv, nullptr, 0);
  SG_DISPATCH(dtype, {
    SG_MASK_DISPATCH(mask_mode, {
      split_sumsq<T, MM>((int)H, (int)W, w, m.as<MM>(), alpha, 1.0 / reciprocal_beta, zero_p, out, as_stream(stream));
    });
  });
  return check_launch("sg_rbsor_split_sumsq");
}

int sg_rbsor_tol_solve(int dtype, int64_t H, int64_t W, void* p, int64_t ld_p, const void* div, int64_t ld_div,
                       int mask_mode, const uint8_t* fmu, int64_t ld_fmu, const uint8_t* fmv, int64_t ld_fmv,
                       double alpha, double reciprocal_beta, double omega, double tol, int64_t max_iterations,
                       int64_t check_every, int variant, void* workspace, int64_t workspace_bytes,
                       int64_t* out_iterations, double* out_relres, void* stream) {
  SplitWs w{};
  SG_CHECK(split_bind(dtype, H, W, workspace, workspace_bytes, &w));
  SG_REQUIRE(p && div && ld_p >= W && ld_div >= W, "bad fields");
  SG_REQUIRE(max_iterations >= 0 && check_every >= 1, "max_iterations >= 0 and check_every >= 1 required");
  SG_REQUIRE(reciprocal_beta != 0.0, "reciprocal_beta must be non-zero");
  SG_REQUIRE(variant >= -1 && variant <= 1, "variant must be -1 (automatic), 0 (half-sweep launches) or 1 (tiles)");
  SG_CHECK(split_mask_check(mask_mode, fmu, fmv));
  Masks m = make_masks(mask_mode, H, W, fmu, ld_fmu, fmv, ld_fmv, nullptr, 0);
  cudaStream_t s = as_stream(stream);
  SG_CHECK(sg_rbsor_split_pack(dtype, H, W, p, ld_p, 0, workspace, workspace_bytes, stream));
  SG_CHECK(sg_rbsor_split_pack(dtype, H, W, div, ld_div, 1, workspace, workspace_bytes, stream));
  int64_t it = 0;
  double rel = 0.0;
  SG_DISPATCH(dtype, {
    const int var = resolve_variant(variant, H, W, sizeof(T));
    SG_MASK_DISPATCH(mask_mode, {
      const MasksT<MM> mm = m.as<MM>();
      const double beta = 1.0 / reciprocal_beta;
      double sq0 = 0.0, sq = 0.0;
      split_sumsq<T, MM>((int)H, (int)W, w, mm, alpha, beta, 1, w.result + 1, s);
      SG_CHECK(check_launch("sg_rbsor_tol_solve"));
      SG_CHECK(read_scalar(w.result + 1, &sq0, s));
      const double r0 = std::sqrt(sq0);
      split_sumsq<T, MM>((int)H, (int)W, w, mm, alpha, beta, 0, w.result, s);
      SG_CHECK(read_scalar(w.result, &sq, s));
      rel = r0 > 0.0 ? std::sqrt(sq) / r0 : 0.0;
      while (rel > tol && it < max_iterations) {
        const int64_t n = std::min(check_every, max_iterations - it);
        SG_CHECK((split_sweeps<T, MM>((int)H, (int)W, w, mm, alpha, reciprocal_beta, omega, n, var, s)));
        it += n;
        split_sumsq<T, MM>((int)H, (int)W, w, mm, alpha, beta, 0, w.result, s);
        SG_CHECK(check_launch("sg_rbsor_tol_solve"));
        SG_CHECK(read_scalar(w.result, &sq, s));
        rel = r0 > 0.0 ? std::sqrt(sq) / r0 : 0.0;
        if (!std::isfinite(rel)) break;
      }
    });
  });
  SG_CHECK(sg_rbsor_split_unpack(dtype, H, W, workspace, workspace_bytes, p, ld_p, stream));
  if (out_iterations) *out_iterations = it;
  if (out_relres) *out_relres = rel;
  if (!std::isfinite(rel)) return fail(SG_ERR_NONFINITE, "non-finite SOR residual after %lld sweeps", (long long)it);
  if (rel > tol)
    return fail(SG_ERR_NOT_CONVERGED, "SOR relative residual %.3e > %.3e after %lld sweeps", rel, tol, (long long)it);
  return SG_OK;
}

int64_t sg_rbsor_mixed_workspace_bytes(int64_t H, int64_t W) {
  if (H < 1 || W < 1) return -1;
  return (int64_t)mixed_bytes(H, W, nullptr, nullptr, nullptr);
}

int sg_rbsor_mixed_solve(int64_t H, int64_t W, void* p, int64_t ld_p, const void* div, int64_t ld_div, int mask_mode,
                         const uint8_t* fmu, int64_t ld_fmu, const uint8_t* fmv, int64_t ld_fmv, double alpha,
                         double reciprocal_beta, double omega, double tol, int64_t max_iterations, int64_t check_every,
                         int variant, void* workspace, int64_t workspace_bytes, int64_t* out_iterations,
                         double* out_relres, int64_t* out_refinements, void* stream) {
  SG_REQUIRE(H >= 1 && W >= 1 && H <= (1 << 28) && W <= (1 << 28), "bad grid %lld x %lld", (long long)H, (long long)W);
  SG_REQUIRE(workspace && !((uintptr_t)workspace & 255), "workspace must be non-null and 256-byte aligned");
  SG_REQUIRE((size_t)workspace_bytes >= mixed_bytes(H, W, nullptr, nullptr, nullptr), "workspace of %lld bytes too small",
             (long long)workspace_bytes);
  SG_REQUIRE(p && div && ld_p >= W && ld_div >= W, "bad fields");
  SG_REQUIRE(max_iterations >= 0 && check_every >= 1, "max_iterations >= 0 and check_every >= 1 required");
  SG_REQUIRE(reciprocal_beta != 0.0, "reciprocal_beta must be non-zero");
  SG_REQUIRE(variant >= -1 && variant <= 1, "variant must be -1 (automatic), 0 (half-sweep launches) or 1 (tiles)");
  SG_CHECK(split_mask_check(mask_mode, fmu, fmv));
  SplitWs w{};
  double* p64 = nullptr;
  mixed_bytes(H, W, &w, &p64, workspace);
  const int var = resolve_variant(variant, H, W, 4);
  Masks m = make_masks(mask_mode, H, W, fmu, ld_fmu, fmv, ld_fmv, nullptr, 0);
  cudaStream_t s = as_stream(stream);
  const double beta = 1.0 / reciprocal_beta;
  const int64_t cells = H * W;
  const int rblocks = (int)std::min<int64_t>(kSumBlocks, (cells + 255) / 256);
  int64_t it = 0, outer = 0;
  double rel = 0.0;
  SG_LAUNCH(k_widen<<<grid2d(W, H), block2d(), 0, s>>>((int)H, (int)W, (const float*)p, ld_p, p64));
  SG_MASK_DISPATCH(mask_mode, {
    const MasksT<MM> mm = m.as<MM>();
    double sq0 = 0.0, sq = 0.0;
    SG_LAUNCH(k_mixed_residual<MM><<<rblocks, 256, 0, s>>>((int)H, (int)W, p64, (const float*)div, ld_div, mm, alpha,
                                                           beta, 1, nullptr, nullptr, w.ldh, w.partials));
    SG_LAUNCH(k_sumsq_finalize<<<1, 256, 0, s>>>(w.partials, rblocks, w.result + 1));
    SG_CHECK(check_launch("sg_rbsor_mixed_solve"));
    SG_CHECK(read_scalar(w.result + 1, &sq0, s));
    const double r0 = std::sqrt(sq0);
    while (true) {
      // outer residual in float64; its float32 rounding becomes the correction's rhs
      SG_LAUNCH(k_mixed_residual<MM><<<rblocks, 256, 0, s>>>((int)H, (int)W, p64, (const float*)div, ld_div, mm, alpha,
                                                             beta, 0, (float*)w.d[0], (float*)w.d[1], w.ldh,
                                                             w.partials));
      SG_LAUNCH(k_sumsq_finalize<<<1, 256, 0, s>>>(w.partials, rblocks, w.result));
      SG_CHECK(check_launch("sg_rbsor_mixed_solve"));
      SG_CHECK(read_scalar(w.result, &sq, s));
      rel = r0 > 0.0 ? std::sqrt(sq) / r0 : 0.0;
      if (!std::isfinite(rel) || rel <= tol || it >= max_iterations) break;
      // inner solve A e = r from e = 0 in float32, to a relative reduction that float32 can
      // reach (1e-3, its floor being ~1e-4) or that the outer target needs, whichever is looser
      const double inner_tol = std::min(0.5, std::max(1e-3, 0.5 * tol / rel));
      for (int c = 0; c < 2; ++c) {
        cudaError_t e = cudaMemsetAsync(w.a[c], 0, w.plane, s);
        if (e != cudaSuccess) return fail(SG_ERR_CUDA, "memset: %s", cudaGetErrorString(e));
      }
      double isq0 = 0.0, isq = 0.0;
      split_sumsq<float, MM>((int)H, (int)W, w, mm, 1.0, beta, 1, w.result + 1, s);
      SG_CHECK(read_scalar(w.result + 1, &isq0, s));
      const double ir0 = std::sqrt(isq0);
      double irel = 1.0, best = 1.0;
      int stalls = 0;
      while (irel > inner_tol && it < max_iterations) {
        const int64_t n = std::min(check_every, max_iterations - it);
        SG_CHECK((split_sweeps<float, MM>((int)H, (int)W, w, mm, 1.0, reciprocal_beta, omega, n, var, s)));
        it += n;
        split_sumsq<float, MM>((int)H, (int)W, w, mm, 1.0, beta, 0, w.result, s);
        SG_CHECK(check_launch("sg_rbsor_mixed_solve"));
        SG_CHECK(read_scalar(w.result, &isq, s));
        irel = ir0 > 0.0 ? std::sqrt(isq) / ir0 : 0.0;
        if (!std::isfinite(irel)) break;
        // float32 floor: stop the inner solve when three chunks in a row gain less than 1 %
        if (irel < 0.99 * best) {
          best = irel;
          stalls = 0;
        } else if (++stalls >= 3) {
          break;
        }
      }
      SG_LAUNCH(k_add_correction<<<grid2d(W, H), block2d(), 0, s>>>((int)H, (int)W, (const float*)w.a[0],
                                                                   (const float*)w.a[1], w.ldh, p64));
      ++outer;
      if (!std::isfinite(irel)) {
        rel = irel;
        break;
      }
    }
  });
  SG_LAUNCH(k_narrow<<<grid2d(W, H), block2d(), 0, s>>>((int)H, (int)W, p64, (float*)p, ld_p));
  SG_CHECK(check_launch("sg_rbsor_mixed_solve"));
  if (out_iterations) *out_iterations = it;
  if (out_relres) *out_relres = rel;
  if (out_refinements) *out_refinements = outer;
  if (!std::isfinite(rel)) return fail(SG_ERR_NONFINITE, "non-finite SOR residual after %lld sweeps", (long long)it);
  if (rel > tol)
    return fail(SG_ERR_NOT_CONVERGED, "mixed SOR relative residual %.3e > %.3e after %lld sweeps", rel, tol,
                (long long)it);
  return SG_OK;
}

}  // extern "C"

SG_BOUNDS_ACCESSOR(rbsor_split)
