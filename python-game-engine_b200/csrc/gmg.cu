// Convergent geometric multigrid (no reference counterpart; the reference V-cycle,
// src/cfd/backends/numba/solvers/multigrid/solver.py, stalls at ~1e-1 relative residual).
//
// Problem: A p = b on fluid cells, A p = sum over open faces (p - p_nb), b = alpha * div,
// so r = b - A p is the reference residual (residual.py:39-40).
// Hierarchy: any-fluid 2x2 coarsening (odd extents round up), faces open between two
// fluid cells. Smoother: red-black Gauss-Seidel, exact diagonal, over-relaxation omega.
// Transfers: bilinear cell-centred prolongation P (clamped to the grid; a non-fluid
// coarse candidate is replaced by the home cell) and full weighting R = P^T, so the
// coarse rhs is P^T r (the factor 4 between A_h and A_2h is absorbed).
// Coarsest level: exact solve with the pseudo-inverse of its operator (host-built).
// Outer loop: residual-correction form r = b - A p (precision of p), e = cycle(r) in the
// cycle precision, p += e; SG_GMG_MIXED runs FP32 cycles inside FP64 refinement.
//
// Execution: levels up to 1024 x 1024 cells in total shared-memory footprint run as one
// thread block (the "tail": every level <= 128^2 in FP32, <= 64^2 in FP64, down to the
// exact coarsest solve) so the launch-latency-bound coarse levels cost one launch per
// visit. Larger levels use grid-wide kernels (zero-initial-guess first sweep and the
// residual fused into the restriction). The tolerance loop is one CUDA graph whose
// cycles sit in a conditional WHILE node; the convergence test runs on the device, so
// a solve needs no host synchronisation.

#include <algorithm>
#include <type_traits>

#include <cooperative_groups.h>
#include <cstring>
#include <vector>

#include "bulk_copy.cuh"
#include "common.cuh"

namespace sg {

// Per-cell code of a level: bit0 fluid, bit1 left face open, bit2 right, bit3 down, bit4 up.
enum : uint8_t { C_FLUID = 1, C_L = 2, C_R = 4, C_D = 8, C_U = 16 };

struct LevelMask {
  const uint8_t* code;  // H x W codes, row stride W (planes mode only)
  int analytic;         // 1: all cells fluid and every interior face open
  int H, W;
  __device__ __forceinline__ uint8_t get(int j, int i) const {
    if (!analytic) return code[(int64_t)j * W + i];
    uint8_t c = C_FLUID;
    if (i > 0) c |= C_L;
    if (i < W - 1) c |= C_R;
    if (j > 0) c |= C_D;
    if (j < H - 1) c |= C_U;
    return c;
  }
  __device__ __forceinline__ bool fluid(int j, int i) const {
    return analytic ? true : (code[(int64_t)j * W + i] & C_FLUID) != 0;
  }
};

constexpr int kHist = 128;  // relative residuals kept per solve (history[0] = initial)

// Solve state in device memory (written by the graph, read by the host on demand).
struct GmgState {
  double bnorm;
  double relres;
  double tol;
  double alpha;
  int cycles;
  int max_cycles;
  int status;  // 0 running, 1 converged, 2 cycle cap reached, 3 non-finite residual, 4 device error
  int dev_error;  // non-zero: a kernel's bounded wait gave up (kDevErr* code); the solve stops
  long long total_cycles;  // cycles run since the plan was bound (all solves)
  long long solves;
  long long failures;      // solves that ended at the cycle cap or on a non-finite residual
  double history[kHist];
  double bmean;  // mean of alpha div over the fluid cells (when the plan removes it)
};

// ---------------------------------------------------------------- point operations
// Residual b - A e at (j, i) of a level (0 on non-fluid cells).
template <typename T>
__device__ __forceinline__ T residual_at(int j, int i, const T* e, int64_t lde, const T* b, int64_t ldb,
                                         const LevelMask& m) {
  uint8_t c = m.get(j, i);
  if (!(c & C_FLUID)) return (T)0;
  int64_t o = (int64_t)j * lde + i;
  T x = e[o];
  T acc = b[(int64_t)j * ldb + i];
  if (c & C_L) acc += e[o - 1] - x;
  if (c & C_R) acc += e[o + 1] - x;
  if (c & C_D) acc += e[o - lde] - x;
  if (c & C_U) acc += e[o + lde] - x;
  return acc;
}

// One Gauss-Seidel update with over-relaxation at (j, i) (no-op on non-fluid / isolated cells).
template <typename T>
__device__ __forceinline__ void relax_at(int j, int i, T* e, int64_t lde, const T* b, int64_t ldb, const LevelMask& m,
                                         T omega) {
  uint8_t c = m.get(j, i);
  if (!(c & C_FLUID)) return;
  int64_t o = (int64_t)j * lde + i;
  T acc = b[(int64_t)j * ldb + i];
  int n = 0;
  if (c & C_L) { acc += e[o - 1]; ++n; }
  if (c & C_R) { acc += e[o + 1]; ++n; }
  if (c & C_D) { acc += e[o - lde]; ++n; }
  if (c & C_U) { acc += e[o + lde]; ++n; }
  if (n == 0) return;
  T x = e[o];
  T gs = acc / (T)n;
  e[o] = x + omega * (gs - x);
}

// Coarse candidates of fine cell (j, i) for bilinear prolongation (weights 9,3,3,1 / 16).
__device__ __forceinline__ void pcand(int j, int i, int Hc, int Wc, const LevelMask& cm, int cj[4], int ci[4]) {
  int J = j >> 1, I = i >> 1;
  int X = I + ((i & 1) ? 1 : -1), Y = J + ((j & 1) ? 1 : -1);
  X = X < 0 ? 0 : (X > Wc - 1 ? Wc - 1 : X);
  Y = Y < 0 ? 0 : (Y > Hc - 1 ? Hc - 1 : Y);
  cj[0] = J; ci[0] = I;
  cj[1] = J; ci[1] = X;
  cj[2] = Y; ci[2] = I;
  cj[3] = Y; ci[3] = X;
#pragma unroll
  for (int q = 1; q < 4; ++q)
    if (!cm.fluid(cj[q], ci[q])) { cj[q] = J; ci[q] = I; }
}

#include "gmg_weights.cuh"

// (P^T r)(J, I) with r evaluated on the fly from e and b of the fine level.
template <typename T>
__device__ __forceinline__ T restrict_at(int J, int I, const T* e, int64_t lde, const T* b, int64_t ldb,
                                         const LevelMask& fm, const LevelMask& cm) {
  int H = fm.H, W = fm.W, Hc = cm.H, Wc = cm.W;
  T acc = (T)0;
  if (fm.analytic && cm.analytic) {
#pragma unroll
    for (int dj = 0; dj < 4; ++dj) {
      int j = 2 * J - 1 + dj;
      if (j < 0 || j >= H) continue;
      T wy = (T)w1(j, J, Hc);
#pragma unroll
      for (int di = 0; di < 4; ++di) {
        int i = 2 * I - 1 + di;
        if (i < 0 || i >= W) continue;
        T w = wy * (T)w1(i, I, Wc);
        if (w != (T)0) acc += w * residual_at(j, i, e, lde, b, ldb, fm);
      }
    }
    return acc;
  }
  if (!cm.fluid(J, I)) return (T)0;
  const T wq[4] = {(T)(9.0 / 16.0), (T)(3.0 / 16.0), (T)(3.0 / 16.0), (T)(1.0 / 16.0)};
  for (int j = 2 * J - 2; j <= 2 * J + 3; ++j) {
    if (j < 0 || j >= H) continue;
    for (int i = 2 * I - 2; i <= 2 * I + 3; ++i) {
      if (i < 0 || i >= W || !fm.fluid(j, i)) continue;
      int cj[4], ci[4];
      pcand(j, i, Hc, Wc, cm, cj, ci);
      T w = (T)0;
#pragma unroll
      for (int q = 0; q < 4; ++q)
        if (cj[q] == J && ci[q] == I) w += wq[q];
      if (w != (T)0) acc += w * residual_at(j, i, e, lde, b, ldb, fm);
    }
  }
  return acc;
}

// (P ec)(j, i) on a fluid fine cell.
template <typename T>
__device__ __forceinline__ T prolong_at(int j, int i, const T* ec, int64_t ldc, const LevelMask& cm) {
  const T wq[4] = {(T)(9.0 / 16.0), (T)(3.0 / 16.0), (T)(3.0 / 16.0), (T)(1.0 / 16.0)};
  int cj[4], ci[4];
  pcand(j, i, cm.H, cm.W, cm, cj, ci);
  T acc = (T)0;
#pragma unroll
  for (int q = 0; q < 4; ++q) acc += wq[q] * ec[(int64_t)cj[q] * ldc + ci[q]];
  return acc;
}

// ---------------------------------------------------------------- grid-wide kernels
// Red-black half sweep. zero_init (first sweep of a zero initial guess, colour 0 only):
// each thread owns the cell pair (2k, 2k+1) of its row, writes the relaxed red cell from
// b alone and zeroes the black one, replacing a separate clearing pass.
template <typename T>
__global__ void k_gmg_rbgs(int H, int W, T* __restrict__ e, int64_t ld, const T* __restrict__ b, LevelMask m, T omega,
                           int color, int zero_init) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (j >= H || 2 * k >= W) return;
  int i = 2 * k + ((j + color) & 1);
  if (zero_init) {
    int i2 = 2 * k + 1 - ((j + color) & 1);
    if (i2 < W) e[(int64_t)j * ld + i2] = (T)0;
    if (i < W) {
      uint8_t c = m.get(j, i);
      int n = __popc(c & (C_L | C_R | C_D | C_U));
      T v = (T)0;
      if ((c & C_FLUID) && n > 0) v = omega * (b[(int64_t)j * ld + i] / (T)n);
      e[(int64_t)j * ld + i] = v;
    }
    return;
  }
  if (i < W) relax_at(j, i, e, ld, b, ld, m, omega);
}

// bc = P^T (b - A e): residual fused into the full-weighting restriction.
template <typename T>
__global__ void k_gmg_residual_restrict(const T* __restrict__ e, const T* __restrict__ b, int64_t ld, LevelMask fm,
                                        T* __restrict__ bc, int64_t ldc, LevelMask cm) {
  int I = blockIdx.x * blockDim.x + threadIdx.x;
  int J = blockIdx.y * blockDim.y + threadIdx.y;
  if (I >= cm.W || J >= cm.H) return;
  bc[(int64_t)J * ldc + I] = restrict_at(J, I, e, ld, b, ld, fm, cm);
}

// e += P ec on fluid fine cells.
template <typename T>
__global__ void k_gmg_prolong_add(const T* __restrict__ ec, int64_t ldc, LevelMask cm, T* __restrict__ e, int64_t lde,
                                  LevelMask fm) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= fm.W || j >= fm.H || !fm.fluid(j, i)) return;
  e[(int64_t)j * lde + i] += prolong_at(j, i, ec, ldc, cm);
}

// Fine residual r = bf - A p in the precision of p, stored as the cycle rhs (TO), with
// per-block sums of r^2.
// Fine-level kernels run 32 x 8 blocks over 128 x 8 cells: each thread takes 4 cells of a
// row, 32 apart, so every load instruction is coalesced and 4 are in flight per thread.
constexpr int kWX = 128;
inline dim3 grid_wide(int64_t W, int64_t H) {
  return dim3((unsigned)((W + kWX - 1) / kWX), (unsigned)((H + kBY - 1) / kBY));
}

template <typename T, typename TO>
__global__ void k_gmg_fine_residual(int H, int W, const T* __restrict__ p, int64_t ldp, const T* __restrict__ bf,
                                    int64_t ldb, LevelMask m, TO* __restrict__ r, int64_t ldr, T* __restrict__ rfull,
                                    double* __restrict__ partial) {
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int ib = blockIdx.x * kWX + threadIdx.x;
  double sq = 0.0;
  if (j < H) {
#pragma unroll
    for (int q = 0; q < kWX / 32; ++q) {
      const int i = ib + 32 * q;
      if (i < W) {
        T acc = residual_at(j, i, p, ldp, bf, ldb, m);
        sq += (double)acc * (double)acc;
        r[(int64_t)j * ldr + i] = (TO)acc;
        if (rfull) rfull[(int64_t)j * ldr + i] = acc;
      }
    }
  }
  double s = block_sum(sq);
  if (threadIdx.x == 0 && threadIdx.y == 0) partial[blockIdx.y * gridDim.x + blockIdx.x] = s;
}

// bf = alpha * div on fluid cells (alpha from the solve state; b may be null when only the
// outputs below are needed) plus per-block sums of bf^2.
// For a zero initial guess (pz non-null) it also writes p = 0 and, bf being the residual,
// the first cycle's rhs b0 (cycle precision) and the carried residual r64 (when kept).
template <typename TD, typename TB, typename TC>
__global__ void k_gmg_rhs(int H, int W, const TD* __restrict__ div, int64_t ldd, const GmgState* __restrict__ st,
                          LevelMask m, TB* __restrict__ b, int64_t ldb, double* __restrict__ partial,
                          TB* __restrict__ pz, int64_t ldpz, TC* __restrict__ b0, int64_t ld0, TB* __restrict__ r64,
                          int sub_mean) {
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int ib = blockIdx.x * kWX + threadIdx.x;
  const double alpha = st->alpha;
  const double mean = sub_mean ? st->bmean : 0.0;
  double sq = 0.0;
  if (j < H) {
#pragma unroll
    for (int q = 0; q < kWX / 32; ++q) {
      const int i = ib + 32 * q;
      if (i < W) {
        TB v = (TB)0;
        if (m.fluid(j, i)) {
          double x = alpha * (double)div[(int64_t)j * ldd + i];
          if (sub_mean) x -= mean;
          v = (TB)x;
          sq += (double)v * (double)v;
        }
        if (b) b[(int64_t)j * ldb + i] = v;
        if (pz) {
          pz[(int64_t)j * ldpz + i] = (TB)0;
          b0[(int64_t)j * ld0 + i] = (TC)v;
          if (r64) r64[(int64_t)j * ld0 + i] = v;
        }
      }
    }
  }
  double s = block_sum(sq);
  if (threadIdx.x == 0 && threadIdx.y == 0) partial[blockIdx.y * gridDim.x + blockIdx.x] = s;
}

// p += e (fine precision += cycle precision).
template <typename TP, typename TE>
__global__ void k_gmg_correct(int H, int W, TP* __restrict__ p, int64_t ldp, const TE* __restrict__ e, int64_t lde) {
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int ib = blockIdx.x * kWX + threadIdx.x;
  if (j >= H) return;
#pragma unroll
  for (int q = 0; q < kWX / 32; ++q) {
    const int i = ib + 32 * q;
    if (i < W) p[(int64_t)j * ldp + i] += (TP)e[(int64_t)j * lde + i];
  }
}

// Sum of partial[0 .. n) over one block (1-D, a multiple of 32 threads): strided sums, then
// warp shuffles and one barrier (a fixed order, so the result is reproducible); the result
// is valid in every thread of warp 0.
__device__ __forceinline__ double sum_partials(const double* __restrict__ partial, int n) {
  double s = 0.0;
  for (int k = threadIdx.x; k < n; k += blockDim.x) s += partial[k];
  s = warp_sum(s);
  __shared__ double red[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) red[warp] = s;
  __syncthreads();
  double t = 0.0;
  if (warp == 0) t = warp_sum(lane < (int)(blockDim.x >> 5) ? red[lane] : 0.0);
  return t;
}

__global__ void k_gmg_set_params(GmgState* st, double alpha, double tol, int max_cycles) {
  st->alpha = alpha;
  st->tol = tol;
  st->max_cycles = max_cycles;
  st->cycles = 0;
  st->status = 0;
  st->solves += 1;
}

// Per-block sums of div over the fluid cells (for the mean the plan removes from the rhs).
template <typename TD>
__global__ void k_gmg_rhs_sum(int H, int W, const TD* __restrict__ div, int64_t ldd, LevelMask m,
                              double* __restrict__ partial) {
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int ib = blockIdx.x * kWX + threadIdx.x;
  double acc = 0.0;
  if (j < H) {
#pragma unroll
    for (int q = 0; q < kWX / 32; ++q) {
      const int i = ib + 32 * q;
      if (i < W && m.fluid(j, i)) acc += (double)div[(int64_t)j * ldd + i];
    }
  }
  double s = block_sum(acc);
  if (threadIdx.x == 0 && threadIdx.y == 0) partial[blockIdx.y * gridDim.x + blockIdx.x] = s;
}

__global__ void k_gmg_finalize_mean(const double* __restrict__ partial, int n, GmgState* st, double inv_fluid) {
  double s = sum_partials(partial, n);
  if (threadIdx.x == 0) st->bmean = st->alpha * (s * inv_fluid);
}

__global__ void k_gmg_finalize_norm(const double* __restrict__ partial, int n, GmgState* st) {
  double s = sum_partials(partial, n);
  if (threadIdx.x == 0) st->bnorm = sqrt(s);
}

// Relative residual after the prologue (body = 0) or a body of `body` cycles; decides whether
// the WHILE node runs another cycle (when use_handle) and records the status.
__device__ void finalize_rel_state(double s, GmgState* st, cudaGraphConditionalHandle h, int use_handle, int body) {
  double nb = st->bnorm;
  double rel = sqrt(s);
  if (!(nb == nb) || isinf(nb)) rel = nb + rel;  // a non-finite ||b|| makes the ratio non-finite
  else rel = nb > 0.0 ? rel / nb : 0.0;
  if (body) {  // body = the number of V/W-cycles the graph body ran
    st->cycles += body;
    st->total_cycles += body;
  }
  int c = st->cycles;
  st->relres = rel;
  if (c < kHist) st->history[c] = rel;
  bool finite = (rel == rel) && !isinf(rel);
  int status = st->dev_error ? 4 : (!finite ? 3 : (rel <= st->tol ? 1 : (c >= st->max_cycles ? 2 : 0)));
  st->status = status;
  if (status >= 2) st->failures += 1;
  if (use_handle) cudaGraphSetConditional(h, status == 0 ? 1u : 0u);
}

__global__ void k_gmg_finalize_rel(const double* __restrict__ partial, int n, GmgState* st, cudaGraphConditionalHandle h,
                                   int use_handle, int body) {
  double s = sum_partials(partial, n);
  if (threadIdx.x == 0) finalize_rel_state(s, st, h, use_handle, body);
}

// ---------------------------------------------------------------- single-block tail
constexpr int kMaxLevels = 16;
constexpr int kPinvMaxSide = 16;  // coarsest levels up to this side: dense pseudo-inverse
constexpr int kDctMaxSide = 64;   // open-box coarsest levels up to this side: one-block cosine transform
constexpr int kDctMultiMaxSide = 256;  // and up to this side: the transform as four tiled products

// Exact solve of an open-box coarsest level by the discrete cosine transform. Its operator
// (sum over open faces of e - e_nb, walls closed) is L_y (x) I + I (x) L_x, L the Laplacian
// of a path of n cells, whose orthonormal eigenvectors are the DCT-II basis
// c_k(i) = s_k cos(pi k (i + 1/2) / n) (s_0 = sqrt(1/n), s_k = sqrt(2/n)) with eigenvalues
// 4 sin^2(pi k / (2 n)). So e = C_y^T [(C_y b C_x^T) / (lambda_y + lambda_x)] C_x with the
// constant mode (0, 0) set to 0, which is the pseudo-inverse solution the dense
// pseudo-inverse gives on smaller coarsest levels. One block of 1024 threads; b and e in the
// level type T, the arithmetic and tab in TA (float64 in mixed precision, as for the dense
// pseudo-inverse; copied whole into shared memory) = C_x (c_k(i) at k W + i), C_x^T,
// C_y (H x H), lambda_x (W), lambda_y (H). Every product keeps four partial sums.
template <typename T, typename TA = T>
__global__ void __launch_bounds__(1024) k_gmg_coarse_dct(const T* __restrict__ b, int64_t ldb, T* __restrict__ e,
                                                         int64_t lde, int H, int W, const TA* __restrict__ tab) {
  extern __shared__ __align__(16) unsigned char dct_smem[];
  TA* sm = reinterpret_cast<TA*>(dct_smem);
  const int ntab = 2 * W * W + H * H + W + H;
  const TA* cx = sm;             // cx[k W + i]
  const TA* cxt = cx + W * W;    // cxt[i W + k]
  const TA* cy = cxt + W * W;    // cy[m H + j]
  const TA* lx = cy + H * H;
  const TA* ly = lx + W;
  TA* X = sm + ntab;
  TA* Y = X + H * W;
  const int tid = threadIdx.x, nt = blockDim.x, n = H * W;
  for (int q = tid; q < ntab; q += nt) sm[q] = tab[q];
  for (int q = tid; q < n; q += nt) {
    const int j = q / W, i = q - j * W;
    Y[q] = (TA)b[(int64_t)j * ldb + i];
  }
  __syncthreads();
  // sum_t a[t * sa] * c[t * sc] over t < len with four partial sums
  auto dot = [](const TA* a, int sa, const TA* c, int sc, int len) {
    TA s0 = (TA)0, s1 = (TA)0, s2 = (TA)0, s3 = (TA)0;
    int t = 0;
    for (; t + 4 <= len; t += 4) {
      s0 += a[t * sa] * c[t * sc];
      s1 += a[(t + 1) * sa] * c[(t + 1) * sc];
      s2 += a[(t + 2) * sa] * c[(t + 2) * sc];
      s3 += a[(t + 3) * sa] * c[(t + 3) * sc];
    }
    for (; t < len; ++t) s0 += a[t * sa] * c[t * sc];
    return (s0 + s1) + (s2 + s3);
  };
  for (int q = tid; q < n; q += nt) {  // X = B C_x^T
    const int j = q / W, k = q - j * W;
    X[q] = dot(Y + j * W, 1, cxt + k, W, W);
  }
  __syncthreads();
  for (int q = tid; q < n; q += nt) {  // Y = (C_y X) / (lambda_y + lambda_x)
    const int m = q / W, k = q - m * W;
    const TA acc = dot(cy + m * H, 1, X + k, W, H);
    Y[q] = (m == 0 && k == 0) ? (TA)0 : acc / (ly[m] + lx[k]);
  }
  __syncthreads();
  for (int q = tid; q < n; q += nt) {  // X = C_y^T Y
    const int j = q / W, k = q - j * W;
    X[q] = dot(cy + j, H, Y + k, W, H);
  }
  __syncthreads();
  for (int q = tid; q < n; q += nt) {  // e = X C_x
    const int j = q / W, i = q - j * W;
    e[(int64_t)j * lde + i] = (T)dot(X + j * W, 1, cx + i, W, W);
  }
}

// The same solve for coarsest levels above kDctMaxSide, as four products over many blocks:
// X = B C_x^T, Y = (C_y X) / (lambda_y + lambda_x) with Y(0, 0) = 0, Z = C_y^T Y, e = Z C_x.
// k_dct_gemm computes C (M x N) = op(A) (M x K) op(B) (K x N) for K <= kDctMultiMaxSide: a
// block of 256 threads owns a 16 x 16 output tile, stages the whole 16 x K panel of op(A) and
// K x 16 panel of op(B) in shared memory with one round of coalesced loads (the latency of
// these small products is the loads', not the arithmetic's), and each thread forms one output
// with four partial sums. op(A)(m, k) is A[m * lda + k], or A[k * lda + m] with TA; op(B)(k, n)
// is B[k * ldb + n], or B[n * ldb + k] with TB. EPI = 1 divides output (m, n) by
// ly[m] + lx[n] and zeroes (0, 0).
constexpr int kDT = 16;      // output tile side
constexpr int kDP = kDT + 1;  // shared-memory pitch of the panels (conflict-free stores)
template <typename T>
static size_t dct_gemm_smem(int K) {
  return (size_t)2 * K * kDP * sizeof(T);
}
template <typename T, bool TA, bool TB, int EPI>
__global__ void __launch_bounds__(kDT* kDT) k_dct_gemm(int M, int N, int K, const T* __restrict__ A, int64_t lda,
                                                       const T* __restrict__ B, int64_t ldb, T* __restrict__ C,
                                                       int64_t ldc, const T* __restrict__ ly, const T* __restrict__ lx) {
  extern __shared__ __align__(16) unsigned char dct_gemm_smem_raw[];
  T* As = reinterpret_cast<T*>(dct_gemm_smem_raw);  // [k][m], pitch kDP
  T* Bs = As + (size_t)K * kDP;                      // [k][n], pitch kDP
  const int m0 = blockIdx.y * kDT, n0 = blockIdx.x * kDT;
  const int tid = threadIdx.x;
  // every load of both panels is issued before the first store (K <= 256: at most 16 per
  // panel and thread), so the block waits for one round trip, not sixteen
  constexpr int kQ = kDctMultiMaxSide / kDT;
  T va[kQ], vb[kQ];
#pragma unroll
  for (int q = 0; q < kQ; ++q) {
    const int e = tid + q * kDT * kDT;
    va[q] = vb[q] = (T)0;
    if (e < kDT * K) {
      // TA: A[k * lda + m], contiguous in m; otherwise A[m * lda + k], contiguous in k
      const int m = TA ? e % kDT : e / K, k = TA ? e / kDT : e % K;
      const int gm = m0 + m;
      if (gm < M) va[q] = TA ? A[(int64_t)k * lda + gm] : A[(int64_t)gm * lda + k];
      const int n = TB ? e / K : e % kDT, k2 = TB ? e % K : e / kDT;
      const int gn = n0 + n;
      if (gn < N) vb[q] = TB ? B[(int64_t)gn * ldb + k2] : B[(int64_t)k2 * ldb + gn];
    }
  }
#pragma unroll
  for (int q = 0; q < kQ; ++q) {
    const int e = tid + q * kDT * kDT;
    if (e < kDT * K) {
      const int m = TA ? e % kDT : e / K, k = TA ? e / kDT : e % K;
      As[k * kDP + m] = va[q];
      const int n = TB ? e / K : e % kDT, k2 = TB ? e % K : e / kDT;
      Bs[k2 * kDP + n] = vb[q];
    }
  }
  __syncthreads();
  const int r = tid / kDT, c = tid % kDT;
  T s0 = (T)0, s1 = (T)0, s2 = (T)0, s3 = (T)0;
  int k = 0;
  for (; k + 4 <= K; k += 4) {
    s0 += As[k * kDP + r] * Bs[k * kDP + c];
    s1 += As[(k + 1) * kDP + r] * Bs[(k + 1) * kDP + c];
    s2 += As[(k + 2) * kDP + r] * Bs[(k + 2) * kDP + c];
    s3 += As[(k + 3) * kDP + r] * Bs[(k + 3) * kDP + c];
  }
  for (; k < K; ++k) s0 += As[k * kDP + r] * Bs[k * kDP + c];
  const int gm = m0 + r, gn = n0 + c;
  if (gm >= M || gn >= N) return;
  T val = (s0 + s1) + (s2 + s3);
  if (EPI == 1) val = (gm == 0 && gn == 0) ? (T)0 : val / (ly[gm] + lx[gn]);
  C[(int64_t)gm * ldc + gn] = val;
}

template <typename T>
static int set_dct_gemm_smem() {
  const int bytes = (int)dct_gemm_smem<T>(kDctMultiMaxSide);
  cudaError_t e = cudaFuncSetAttribute(k_dct_gemm<T, false, true, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_dct_gemm<T, false, false, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_dct_gemm<T, true, false, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_dct_gemm<T, false, false, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  return e == cudaSuccess ? SG_OK : fail(SG_ERR_CUDA, "cosine-transform products: %s", cudaGetErrorString(e));
}

// The same solve in two launches that stream the operands through shared memory, for
// coarsest levels whose rows are whole 16-byte units (W * sizeof(T) % 16 == 0):
//   forward (one block per kDsRB spectral rows m): T1 = C_y[m, :] B, T2 = T1 C_x^T,
//     Y = T2 / (lambda_y[m] + lambda_x) with Y(0, 0) = 0, X[m, :] = Y C_x;
//   inverse (one block per kDsRB output rows j): e[j, :] = sum_m C_y[m, j] X[m, :].
// Every product here has one streamed operand whose rows are W long (B, C_x^T, C_x, X) and a
// small left factor held in shared memory ([k][r], the block's kDsRB rows side by side), so a
// launch is one stream of rows: warp 0 issues bulk copies of kDsKC rows per chunk into a ring
// of `ns` slots sized to keep most of the stream in flight. A thread owns one column c and
// all kDsRB rows (one vector load of the left factor feeds kDsRB FMAs); the NKG thread groups
// of a block take every NKG-th streamed row and their partial sums meet in shared memory at
// the end of each product. The four products of k_dct_gemm become two launches, and the
// intermediates T1 / T2 never leave shared memory. A wait that gives up sets st->dev_error.
constexpr int kDsRB = 4;                   // rows per block
constexpr int kDsKC = 32;                  // streamed rows per chunk
constexpr int kDsMaxSlots = 32;            // mbarriers reserved at the start of shared memory
constexpr int kDsSmemBudget = 220 * 1024;  // bytes of shared memory per block
constexpr int kDevErrBulkWait = 1;

struct DctStreamLayout {
  int ns;           // ring slots
  size_t off_left;  // left factors: L0 (max(H, W) x kDsRB), L1 and L2 (W x kDsRB)
  size_t off_red;   // partial sums of the thread groups: 3 x kDsRB x W
  size_t off_ring;  // ns x kDsKC x W
  size_t bytes;
};

// The ring takes what the budget leaves: when the whole stream fits (float32 up to ~128^2),
// every chunk has its own slot and the launch needs no slot reuse and no per-chunk barrier.
template <typename T>
__host__ __device__ inline DctStreamLayout dct_stream_layout(int H, int W) {
  DctStreamLayout L;
  const size_t slot = (size_t)kDsKC * W * sizeof(T);
  const int chunks = (H + kDsKC - 1) / kDsKC + 2 * ((W + kDsKC - 1) / kDsKC);
  L.off_left = 8 * kDsMaxSlots;
  L.off_red = L.off_left + ((size_t)(H > W ? H : W) + 2 * (size_t)W) * kDsRB * sizeof(T);
  L.off_ring = (L.off_red + (size_t)3 * kDsRB * W * sizeof(T) + 127) & ~(size_t)127;
  const size_t room = kDsSmemBudget > L.off_ring ? kDsSmemBudget - L.off_ring : 0;
  int ns = (int)(room / slot);
  ns = ns < 2 ? 2 : ns;
  ns = ns > chunks ? chunks : ns;
  ns = ns > kDsMaxSlots ? kDsMaxSlots : ns;
  L.ns = ns;
  L.bytes = L.off_ring + (size_t)ns * slot;
  return L;
}

template <typename T>
__device__ __forceinline__ void load_rows4(const T* __restrict__ p, T (&v)[kDsRB]) {
  static_assert(kDsRB == 4, "four rows per block");
  if constexpr (sizeof(T) == 4) {
    const float4 q = *reinterpret_cast<const float4*>(p);
    v[0] = q.x, v[1] = q.y, v[2] = q.z, v[3] = q.w;
  } else {
    const double2 q0 = *reinterpret_cast<const double2*>(p);
    const double2 q1 = *reinterpret_cast<const double2*>(p + 2);
    v[0] = q0.x, v[1] = q0.y, v[2] = q1.x, v[3] = q1.y;
  }
}

// One chunk's products for the thread's column c: acc[r] += left[t][r] * slot[t][c] over the
// chunk's rows t taken by thread group kg (every NKG-th), slot rows W long in type TS.
template <int NKG, typename TS, typename TA>
__device__ __forceinline__ void dct_stream_consume(const TS* __restrict__ slot, int W, int c, int kg, int nr,
                                                   const TA* __restrict__ left, TA (&acc)[kDsRB]) {
  if (nr == kDsKC) {
#pragma unroll
    for (int tt = 0; tt < kDsKC / NKG; ++tt) {
      const int t = tt * NKG + kg;
      const TA v = (TA)slot[(size_t)t * W + c];
      TA l[kDsRB];
      load_rows4(left + t * kDsRB, l);
#pragma unroll
      for (int r = 0; r < kDsRB; ++r) acc[r] += l[r] * v;
    }
  } else {
    for (int t = kg; t < nr; t += NKG) {
      const TA v = (TA)slot[(size_t)t * W + c];
      TA l[kDsRB];
      load_rows4(left + t * kDsRB, l);
#pragma unroll
      for (int r = 0; r < kDsRB; ++r) acc[r] += l[r] * v;
    }
  }
}

// NKG thread groups of roundup32(W) threads (blockDim = NKG * roundup32(W) <= 256). INVERSE:
// the second launch. b: the level's rhs (row stride ldb) and e its solution, in the level type
// T; the arithmetic, the tables of k_gmg_coarse_dct (tab) and the H x W scratch X (row stride
// W) in TA (float64 in mixed precision).
template <typename T, typename TA, int NKG, bool INVERSE>
__global__ void __launch_bounds__(256, 1) k_dct_stream(int H, int W, const T* __restrict__ b, int64_t ldb,
                                                    const TA* __restrict__ tab, TA* __restrict__ X, T* __restrict__ e,
                                                    int64_t lde, GmgState* __restrict__ st) {
  extern __shared__ __align__(128) unsigned char ds_smem[];
  const DctStreamLayout lay = dct_stream_layout<TA>(H, W);
  uint64_t* full = reinterpret_cast<uint64_t*>(ds_smem);
  TA* L0 = reinterpret_cast<TA*>(ds_smem + lay.off_left);  // [k][r], k < max(H, W)
  TA* L1 = L0 + (size_t)(H > W ? H : W) * kDsRB;           // [i][r], i < W
  TA* L2 = L1 + (size_t)W * kDsRB;                         // [k][r], k < W
  TA* red = reinterpret_cast<TA*>(ds_smem + lay.off_red);  // [group - 1][r][c]
  TA* ring = reinterpret_cast<TA*>(ds_smem + lay.off_ring);  // slots of kDsKC x W elements of TA
  const TA* cx = tab;                   // cx[k W + i]
  const TA* cxt = cx + (int64_t)W * W;  // cxt[i W + k]
  const TA* cy = cxt + (int64_t)W * W;  // cy[m H + j]
  const TA* lx = cy + (int64_t)H * H;
  const TA* ly = lx + W;
  const int tid = threadIdx.x, nt = blockDim.x;
  const int cw = (W + 31) & ~31;
  const int c = tid % cw, kg = tid / cw;  // column and thread group
  const int r0 = blockIdx.x * kDsRB;      // the block's first row (m forward, j inverse)
  const int ns = lay.ns;
  // phases: forward streams B (H rows), C_x^T (W rows), C_x (W rows); inverse streams X (H)
  auto nrows = [&](int q) { return q == 0 ? H : W; };
  auto nch = [&](int q) { return (nrows(q) + kDsKC - 1) / kDsKC; };
  const int total = INVERSE ? nch(0) : nch(0) + 2 * nch(1);
  // warp 0: chunk ch into slot ch % ns. Lane 0 arrives with the chunk's byte count; the
  // copies (one for a contiguous chunk, else one per row from lanes 0 .. nr - 1) may land
  // before that arrival: the phase cannot complete while the arrival is pending.
  auto issue = [&](int ch) {
    const int lane = tid & 31;
    int q = 0, k = ch;
    while (k >= nch(q)) k -= nch(q++);
    const int row0 = k * kDsKC;
    const int nr = min(kDsKC, nrows(q) - row0);
    const bool lvl = !INVERSE && q == 0;  // rows of the level (type T), else of TA
    const unsigned char* src =
        lvl ? reinterpret_cast<const unsigned char*>(b)
            : reinterpret_cast<const unsigned char*>(INVERSE ? (const TA*)X : (q == 1 ? cxt : cx));
    const uint32_t rb = (uint32_t)W * (uint32_t)(lvl ? sizeof(T) : sizeof(TA));
    const int64_t ldbytes = lvl ? ldb * (int64_t)sizeof(T) : (int64_t)rb;
    uint64_t* bar = full + ch % ns;
    unsigned char* dst = reinterpret_cast<unsigned char*>(ring + (size_t)(ch % ns) * kDsKC * W);
    if (lane == 0) mbar_arrive_expect_tx(bar, (uint32_t)nr * rb);
    if (ldbytes == (int64_t)rb) {
      if (lane == 0) bulk_g2s(dst, src + (int64_t)row0 * rb, (uint32_t)nr * rb, bar);
    } else if (lane < nr) {
      bulk_g2s(dst + (size_t)lane * rb, src + (int64_t)(row0 + lane) * ldbytes, rb, bar);
    }
  };
  if (tid == 0) {
    for (int s = 0; s < ns; ++s) mbar_init(full + s, 1);
    mbar_fence_init();
  }
  __syncthreads();
  if (tid < 32)
    for (int ch = 0; ch < ns && ch < total; ++ch) issue(ch);
  // the first left factor: forward C_y[r0 + r, j] at L0[j][r]; inverse C_y[m, r0 + r] at L0[m][r]
  for (int q = tid; q < H * kDsRB; q += nt) {
    const int k = q / kDsRB, r = q - k * kDsRB;
    const int row = r0 + r;
    L0[q] = row < H ? (INVERSE ? cy[(int64_t)k * H + row] : cy[(int64_t)row * H + k]) : (TA)0;
  }
  __syncthreads();
  bool ok = true;
  TA acc[kDsRB];
#pragma unroll
  for (int r = 0; r < kDsRB; ++r) acc[r] = (TA)0;
  int q = 0, kq = 0;  // phase of the current chunk and its index within the phase
  for (int ch = 0; ch < total; ++ch) {
    if (!mbar_wait(full + ch % ns, (uint32_t)((ch / ns) & 1))) ok = false;
    const int row0 = kq * kDsKC;
    const int nr = min(kDsKC, nrows(q) - row0);
    const TA* left = (q == 0 ? L0 : (q == 1 ? L1 : L2)) + (size_t)row0 * kDsRB;
    const TA* slot = ring + (size_t)(ch % ns) * kDsKC * W;
    if (c < W) {
      if (!INVERSE && q == 0 && !std::is_same<T, TA>::value)
        dct_stream_consume<NKG>(reinterpret_cast<const T*>(slot), W, c, kg, nr, left, acc);
      else
        dct_stream_consume<NKG>(slot, W, c, kg, nr, left, acc);
    }
    if (++kq == nch(q)) {  // the phase's products are complete: sum the groups, epilogue
      if (NKG > 1) {
        if (kg > 0 && c < W) {
#pragma unroll
          for (int r = 0; r < kDsRB; ++r) red[((size_t)(kg - 1) * kDsRB + r) * W + c] = acc[r];
        }
        __syncthreads();
      }
      if (kg == 0 && c < W) {
#pragma unroll
        for (int r = 0; r < kDsRB; ++r) {
          TA v = acc[r];
#pragma unroll
          for (int g = 1; g < NKG; ++g) v += red[((size_t)(g - 1) * kDsRB + r) * W + c];
          const int row = r0 + r;
          if (INVERSE) {
            if (row < H) e[(int64_t)row * lde + c] = (T)v;
          } else if (q == 0) {
            L1[c * kDsRB + r] = v;
          } else if (q == 1) {
            L2[c * kDsRB + r] = (row == 0 && c == 0) || row >= H ? (TA)0 : v / (ly[row < H ? row : 0] + lx[c]);
          } else if (row < H) {
            X[(int64_t)row * W + c] = v;
          }
        }
      }
#pragma unroll
      for (int r = 0; r < kDsRB; ++r) acc[r] = (TA)0;
      ++q;
      kq = 0;
    }
    if (kq == 0 || ns < total) __syncthreads();  // a left factor written / the slot consumed
    if (tid < 32 && ch + ns < total) issue(ch + ns);
  }
  if (!ok) {
    atomicExch(&st->dev_error, kDevErrBulkWait);
    // let copies still in flight land before the block's shared memory is released
    for (int ch = total - ns < 0 ? 0 : total - ns; ch < total; ++ch) mbar_wait(full + ch % ns, (uint32_t)((ch / ns) & 1));
  }
}

// The streaming transform on thread-block clusters of kDcNC CTAs, for coarsest levels whose
// whole per-CTA stream fits in shared memory (the 2048^2 workload's 128^2 level). One SM's
// intake of its stream bounds k_dct_stream, so here the CTAs of a cluster split every product
// and each streams a kDcNC-th of its operand, in contiguous rows:
//   forward  T1 = C_y[m, :] B      CTA c streams B rows j in its share (partial sums over j),
//            T2 = T1 C_x^T         CTA c forms the output columns k in its share from the split
//                                  table (each of its rows W / kDcNC long),
//            Y  = T2 / (ly + lx)   on those columns,
//            X  = Y C_x            CTA c streams the C_x rows k it holds Y for (partial sums);
//   inverse  e  = C_y^T X          CTA c streams X rows m in its share (partial sums).
// Partial sums meet in distributed shared memory: each CTA publishes its partial, the cluster
// synchronises, and every CTA adds the kDcNC partials in rank order (so all hold the same
// bits of T1); X and e are written by column shares. Rows, chunks and waits as in
// k_dct_stream, except that every chunk has its own place in shared memory.
constexpr int kDcNC = 4;

struct DctClusterLayout {
  int nch;          // chunks in the stream
  size_t off_left;  // L0 (H / kDcNC x kDsRB), L1 (W x kDsRB), L2 (W / kDcNC x kDsRB)
  size_t off_red;   // thread-group partials: 3 x kDsRB x W
  size_t off_xch;   // the CTA's published partial: kDsRB x W
  size_t off_ring;  // the whole stream
  size_t bytes;
};

// Phase q of a launch: rows streamed, bytes per row (level rows are T, the rest TA).
__host__ __device__ inline void dct_cluster_phase(bool inverse, int q, int H, int W, size_t sT, size_t sTA, int& rows,
                                                  size_t& rb) {
  const int hc = H / kDcNC, wc = W / kDcNC;
  if (inverse) {
    rows = hc;
    rb = (size_t)W * sTA;
  } else if (q == 0) {
    rows = hc;
    rb = (size_t)W * sT;
  } else if (q == 1) {
    rows = W;
    rb = (size_t)wc * sTA;
  } else {
    rows = wc;
    rb = (size_t)W * sTA;
  }
}

__host__ __device__ inline DctClusterLayout dct_cluster_layout(bool inverse, int H, int W, size_t sT, size_t sTA) {
  DctClusterLayout L;
  const int nph = inverse ? 1 : 3;
  size_t ring = 0;
  int nch = 0;
  for (int q = 0; q < nph; ++q) {
    int rows;
    size_t rb;
    dct_cluster_phase(inverse, q, H, W, sT, sTA, rows, rb);
    ring += (size_t)rows * rb;
    nch += (rows + kDsKC - 1) / kDsKC;
  }
  L.nch = nch;
  L.off_left = 8 * kDsMaxSlots;
  L.off_red = L.off_left + ((size_t)H / kDcNC + (size_t)W + (size_t)W / kDcNC) * kDsRB * sTA;
  L.off_xch = L.off_red + (size_t)3 * kDsRB * W * sTA;
  L.off_ring = (L.off_xch + (size_t)kDsRB * W * sTA + 127) & ~(size_t)127;
  L.bytes = L.off_ring + ring;
  return L;
}

template <typename T, typename TA, int NKG, bool INVERSE>
__global__ void __cluster_dims__(kDcNC, 1, 1) __launch_bounds__(256, 1)
    k_dct_cluster(int H, int W, const T* __restrict__ b, int64_t ldb, const TA* __restrict__ tab, TA* __restrict__ X,
                  T* __restrict__ e, int64_t lde, GmgState* __restrict__ st) {
  namespace cg = cooperative_groups;
  extern __shared__ __align__(128) unsigned char dc_smem[];
  cg::cluster_group cl = cg::this_cluster();
  const int crank = (int)cl.block_rank();
  const DctClusterLayout lay = dct_cluster_layout(INVERSE, H, W, sizeof(T), sizeof(TA));
  const int hc = H / kDcNC, wc = W / kDcNC;
  uint64_t* full = reinterpret_cast<uint64_t*>(dc_smem);
  TA* L0 = reinterpret_cast<TA*>(dc_smem + lay.off_left);  // [k][r], k < hc
  TA* L1 = L0 + (size_t)hc * kDsRB;                        // [i][r], i < W
  TA* L2 = L1 + (size_t)W * kDsRB;                         // [kl][r], kl < wc
  TA* red = reinterpret_cast<TA*>(dc_smem + lay.off_red);  // [group - 1][r][c]
  TA* xch = reinterpret_cast<TA*>(dc_smem + lay.off_xch);  // [r][c]
  unsigned char* ring = dc_smem + lay.off_ring;
  const TA* cx = tab;                          // cx[k W + i]
  const TA* cy = cx + 2 * (int64_t)W * W;      // cy[m H + j]
  const TA* lx = cy + (int64_t)H * H;
  const TA* ly = lx + W;
  const TA* cxs = ly + H;                      // C_x^T split by output columns
  const int tid = threadIdx.x, nt = blockDim.x;
  const int cw = (W + 31) & ~31;
  const int c = tid % cw, kg = tid / cw;       // column and thread group
  const int r0 = (blockIdx.x / kDcNC) * kDsRB; // the cluster's first row (m forward, j inverse)
  const int nph = INVERSE ? 1 : 3;
  // source of phase q for this CTA, its row stride in bytes and its row length in elements
  auto phase_src = [&](int q, const unsigned char*& src, int64_t& ldbytes, int& rowlen) {
    if (INVERSE) {
      src = reinterpret_cast<const unsigned char*>(X + (int64_t)crank * hc * W);
      ldbytes = (int64_t)W * sizeof(TA);
      rowlen = W;
    } else if (q == 0) {
      src = reinterpret_cast<const unsigned char*>(b + (int64_t)crank * hc * ldb);
      ldbytes = ldb * (int64_t)sizeof(T);
      rowlen = W;
    } else if (q == 1) {
      src = reinterpret_cast<const unsigned char*>(cxs + (int64_t)crank * W * wc);
      ldbytes = (int64_t)wc * sizeof(TA);
      rowlen = wc;
    } else {
      src = reinterpret_cast<const unsigned char*>(cx + (int64_t)crank * wc * W);
      ldbytes = (int64_t)W * sizeof(TA);
      rowlen = W;
    }
  };
  if (tid == 0) {
    for (int k = 0; k < lay.nch; ++k) mbar_init(full + k, 1);
    mbar_fence_init();
  }
  __syncthreads();
  if (tid < 32) {  // warp 0 issues the whole stream (every chunk has its own place)
    const int lane = tid;
    size_t off = 0;
    int ch = 0;
    for (int q = 0; q < nph; ++q) {
      int rows;
      size_t rb;
      dct_cluster_phase(INVERSE, q, H, W, sizeof(T), sizeof(TA), rows, rb);
      const unsigned char* src;
      int64_t ldbytes;
      int rowlen;
      phase_src(q, src, ldbytes, rowlen);
      for (int row0 = 0; row0 < rows; row0 += kDsKC, ++ch) {
        const int nr = min(kDsKC, rows - row0);
        if (lane == 0) mbar_arrive_expect_tx(full + ch, (uint32_t)(nr * rb));
        if (ldbytes == (int64_t)rb) {
          if (lane == 0) bulk_g2s(ring + off, src + (int64_t)row0 * rb, (uint32_t)(nr * rb), full + ch);
        } else if (lane < nr) {
          bulk_g2s(ring + off + (size_t)lane * rb, src + (int64_t)(row0 + lane) * ldbytes, (uint32_t)rb, full + ch);
        }
        off += (size_t)nr * rb;
      }
    }
  }
  // the first left factor: forward C_y[r0 + r, crank hc + j] at L0[j][r]; inverse
  // C_y[crank hc + m, r0 + r] at L0[m][r]
  for (int q = tid; q < hc * kDsRB; q += nt) {
    const int k = q / kDsRB, r = q - k * kDsRB;
    const int row = r0 + r, kk = crank * hc + k;
    L0[q] = row < H ? (INVERSE ? cy[(int64_t)kk * H + row] : cy[(int64_t)row * H + kk]) : (TA)0;
  }
  __syncthreads();
  bool ok = true;
  TA acc[kDsRB];
#pragma unroll
  for (int r = 0; r < kDsRB; ++r) acc[r] = (TA)0;
  size_t off = 0;
  int ch = 0;
  for (int q = 0; q < nph; ++q) {
    int rows;
    size_t rb;
    dct_cluster_phase(INVERSE, q, H, W, sizeof(T), sizeof(TA), rows, rb);
    const unsigned char* src;
    int64_t ldbytes;
    int rowlen;
    phase_src(q, src, ldbytes, rowlen);
    const TA* left = q == 0 ? L0 : (q == 1 ? L1 : L2);
    for (int row0 = 0; row0 < rows; row0 += kDsKC, ++ch) {
      const int nr = min(kDsKC, rows - row0);
      if (!mbar_wait(full + ch, 0)) ok = false;
      if (c < rowlen) {
        if (!INVERSE && q == 0 && !std::is_same<T, TA>::value)
          dct_stream_consume<NKG>(reinterpret_cast<const T*>(ring + off), rowlen, c, kg, nr, left + row0 * kDsRB, acc);
        else
          dct_stream_consume<NKG>(reinterpret_cast<const TA*>(ring + off), rowlen, c, kg, nr, left + row0 * kDsRB,
                                  acc);
      }
      off += (size_t)nr * rb;
    }
    // the phase's products are complete: sum the thread groups
    if (NKG > 1) {
      if (kg > 0 && c < rowlen) {
#pragma unroll
        for (int r = 0; r < kDsRB; ++r) red[((size_t)(kg - 1) * kDsRB + r) * W + c] = acc[r];
      }
      __syncthreads();
    }
    TA v[kDsRB];
#pragma unroll
    for (int r = 0; r < kDsRB; ++r) {
      v[r] = acc[r];
      acc[r] = (TA)0;
      if (kg == 0 && c < rowlen) {
#pragma unroll
        for (int g = 1; g < NKG; ++g) v[r] += red[((size_t)(g - 1) * kDsRB + r) * W + c];
      }
    }
    const bool partial = INVERSE || q != 1;  // sums over a share of the contraction
    if (partial) {  // publish, synchronise the cluster, add the partials in rank order
      if (kg == 0 && c < W) {
#pragma unroll
        for (int r = 0; r < kDsRB; ++r) xch[(size_t)r * W + c] = v[r];
      }
      cl.sync();
      if (kg == 0 && c < W) {
#pragma unroll
        for (int r = 0; r < kDsRB; ++r) v[r] = (TA)0;
        for (int rk = 0; rk < kDcNC; ++rk) {
          const TA* px = cl.map_shared_rank(xch, rk);
#pragma unroll
          for (int r = 0; r < kDsRB; ++r) v[r] += px[(size_t)r * W + c];
        }
      }
      cl.sync();  // every CTA has read the partials before any overwrites its own
    }
    if (kg == 0) {
#pragma unroll
      for (int r = 0; r < kDsRB; ++r) {
        const int row = r0 + r;
        if (INVERSE) {
          if (c < W && c / wc == crank && row < H) e[(int64_t)row * lde + c] = (T)v[r];
        } else if (q == 0) {
          if (c < W) L1[c * kDsRB + r] = v[r];
        } else if (q == 1) {
          if (c < wc) {
            const int k = crank * wc + c;
            L2[c * kDsRB + r] = (row == 0 && k == 0) || row >= H ? (TA)0 : v[r] / (ly[row < H ? row : 0] + lx[k]);
          }
        } else if (c < W && c / wc == crank && row < H) {
          X[(int64_t)row * W + c] = v[r];
        }
      }
    }
    __syncthreads();  // the next phase's left factor is written
  }
  if (!ok) {
    atomicExch(&st->dev_error, kDevErrBulkWait);
    for (int k = 0; k < lay.nch; ++k) mbar_wait(full + k, 0);
  }
}

template <typename T>
static size_t coarse_dct_smem(int H, int W) {
  return (size_t)(2 * W * W + H * H + W + H + 2 * H * W) * sizeof(T);
}

// The tables of k_gmg_coarse_dct for an H x W level (host, double): C_x, C_x^T, C_y,
// lambda_x, lambda_y.
static void coarse_dct_tables(int H, int W, std::vector<double>& tab) {
  const double pi = 3.14159265358979323846;
  tab.assign(2 * (size_t)W * W + (size_t)H * H + W + H, 0.0);
  auto basis = [&](int n, double* c, double* lam) {
    for (int k = 0; k < n; ++k) {
      const double sk = std::sqrt((k == 0 ? 1.0 : 2.0) / n);
      for (int i = 0; i < n; ++i) c[(size_t)k * n + i] = sk * std::cos(pi * k * (i + 0.5) / n);
      const double sn = std::sin(pi * k / (2.0 * n));
      lam[k] = 4.0 * sn * sn;
    }
  };
  double* cx = tab.data();
  double* cxt = cx + (size_t)W * W;
  double* cy = cxt + (size_t)W * W;
  double* lx = cy + (size_t)H * H;
  double* ly = lx + W;
  basis(W, cx, lx);
  basis(H, cy, ly);
  for (int k = 0; k < W; ++k)
    for (int i = 0; i < W; ++i) cxt[(size_t)i * W + k] = cx[(size_t)k * W + i];
}

// The same tables followed by C_x^T split by output columns for a cluster of nc CTAs
// (k_dct_cluster): part c holds cxt[i][c W / nc + kl] at c W (W / nc) + i (W / nc) + kl, so each
// CTA's share of the product T1 C_x^T is one contiguous block of rows.
static void coarse_dct_tables_split(int H, int W, int nc, std::vector<double>& tab) {
  coarse_dct_tables(H, W, tab);
  const size_t base = tab.size();
  const int wc = W / nc;
  tab.resize(base + (size_t)W * W, 0.0);
  const double* cxt = tab.data() + (size_t)W * W;
  double* sp = tab.data() + base;
  for (int c = 0; c < nc; ++c)
    for (int i = 0; i < W; ++i)
      for (int kl = 0; kl < wc; ++kl)
        sp[(size_t)c * W * wc + (size_t)i * wc + kl] = cxt[(size_t)i * W + c * wc + kl];
}
// Levels up to this many cells a side run inside the single-block tail kernel; larger
// open-box levels use the fused tiled kernels (two launches per level and cycle).
constexpr int kTailMaxSide = 16;
constexpr int kTailThreads = 1024;

template <typename T>
struct TailArgs {
  int n;                    // tail levels; the last one is the coarsest (exact solve)
  LevelMask m[kMaxLevels];  // masks (codes in global memory)
  int off_e[kMaxLevels];    // shared-memory offsets (elements of T), row stride = W
  int off_b[kMaxLevels];
  int off_x;                // restriction scratch: rows x coarse columns of the first level
  T* ge;                    // first tail level in global memory (e in/out, b in)
  const T* gb;
  int64_t gld;
  const double* pinv;       // coarsest pseudo-inverse
  T omega;
  int pre, post, wcycle, zero_init;
};


// Open-face bits of (j, i): analytic levels from the bounds, others from their codes.
__device__ __forceinline__ uint8_t tail_code(const LevelMask& m, int j, int i) {
  if (!m.analytic) return m.code[j * m.W + i];
  return (uint8_t)(C_FLUID | (i > 0 ? C_L : 0) | (i < m.W - 1 ? C_R : 0) | (j > 0 ? C_D : 0) | (j < m.H - 1 ? C_U : 0));
}

// Half sweep over shared-memory arrays (row stride W); threads laid out 32 x 32.
template <typename T>
__device__ void tail_relax(const LevelMask& m, T* e, const T* b, T omega, int color) {
  const int H = m.H, W = m.W, Wh = (W + 1) >> 1;
  for (int j = threadIdx.y; j < H; j += blockDim.y) {
    const int par = (j + color) & 1;
    for (int k = threadIdx.x; k < Wh; k += blockDim.x) {
      const int i = 2 * k + par;
      if (i >= W) continue;
      const uint8_t c = tail_code(m, j, i);
      if (!(c & C_FLUID)) continue;
      const int o = j * W + i;
      T acc = b[o];
      int n = 0;
      if (c & C_L) { acc += e[o - 1]; ++n; }
      if (c & C_R) { acc += e[o + 1]; ++n; }
      if (c & C_D) { acc += e[o - W]; ++n; }
      if (c & C_U) { acc += e[o + W]; ++n; }
      if (n == 0) continue;
      const T x = e[o];
      e[o] = x + omega * (acc * rcp_open<T>(n) - x);
    }
  }
  __syncthreads();
}

// Residual b - A e at (j, i) of a shared-memory level.
template <typename T>
__device__ __forceinline__ T tail_res(const LevelMask& m, const T* e, const T* b, int j, int i) {
  const uint8_t c = tail_code(m, j, i);
  if (!(c & C_FLUID)) return (T)0;
  const int W = m.W, o = j * W + i;
  const T x = e[o];
  T acc = b[o];
  if (c & C_L) acc += e[o - 1] - x;
  if (c & C_R) acc += e[o + 1] - x;
  if (c & C_D) acc += e[o - W] - x;
  if (c & C_U) acc += e[o + W] - x;
  return acc;
}

// bc = P^T (b - A e), ec = 0. Analytic level pairs use the separable form: rows of the
// fine level are first restricted along x into the scratch X (H x Wc), then along y.
template <typename T>
__device__ void tail_restrict(const LevelMask& m, const T* e, const T* b, const LevelMask& cm, T* bc, T* ec, T* X) {
  const int H = m.H, W = m.W, Hc = cm.H, Wc = cm.W;
  if (m.analytic && cm.analytic) {
    for (int j = threadIdx.y; j < H; j += blockDim.y)
      for (int I = threadIdx.x; I < Wc; I += blockDim.x) {
        T acc = (T)0;
#pragma unroll
        for (int d = 0; d < 4; ++d) {
          const int i = 2 * I - 1 + d;
          if (i < 0 || i >= W) continue;
          const T w = (T)w1(i, I, Wc);
          if (w != (T)0) acc += w * tail_res(m, e, b, j, i);
        }
        X[j * Wc + I] = acc;
      }
    __syncthreads();
    for (int J = threadIdx.y; J < Hc; J += blockDim.y)
      for (int I = threadIdx.x; I < Wc; I += blockDim.x) {
        T acc = (T)0;
#pragma unroll
        for (int d = 0; d < 4; ++d) {
          const int j = 2 * J - 1 + d;
          if (j < 0 || j >= H) continue;
          const T w = (T)w1(j, J, Hc);
          if (w != (T)0) acc += w * X[j * Wc + I];
        }
        bc[J * Wc + I] = acc;
        ec[J * Wc + I] = (T)0;
      }
  } else {
    for (int J = threadIdx.y; J < Hc; J += blockDim.y)
      for (int I = threadIdx.x; I < Wc; I += blockDim.x) {
        bc[J * Wc + I] = restrict_at(J, I, e, (int64_t)W, b, (int64_t)W, m, cm);
        ec[J * Wc + I] = (T)0;
      }
  }
  __syncthreads();
}

// e += P ec on the fluid cells of a shared-memory level.
template <typename T>
__device__ void tail_prolong(const LevelMask& m, T* e, const LevelMask& cm, const T* ec) {
  for (int j = threadIdx.y; j < m.H; j += blockDim.y)
    for (int i = threadIdx.x; i < m.W; i += blockDim.x)
      if (m.fluid(j, i)) e[j * m.W + i] += prolong_at(j, i, ec, (int64_t)cm.W, cm);
  __syncthreads();
}

template <typename T>
__device__ void tail_coarse_solve(const LevelMask& m, T* e, const T* b, const double* __restrict__ pinv) {
  int n = m.H * m.W;
  int tid = threadIdx.y * blockDim.x + threadIdx.x;
  int lane = tid & 31, warp = tid >> 5, nw = (blockDim.x * blockDim.y) >> 5;
  for (int row = warp; row < n; row += nw) {
    double acc = 0.0;
    for (int q = lane; q < n; q += 32) acc += pinv[(int64_t)row * n + q] * (double)b[q];
    acc = warp_sum(acc);
    if (lane == 0) e[row] = (T)acc;
  }
  __syncthreads();
}

template <typename T>
__device__ __noinline__ void tail_cycle(const TailArgs<T>& a, T* sm, int k) {
  const LevelMask& m = a.m[k];
  T* e = sm + a.off_e[k];
  T* b = sm + a.off_b[k];
  if (k == a.n - 1) {
    tail_coarse_solve(m, e, b, a.pinv);
    return;
  }
  for (int s = 0; s < a.pre; ++s) {
    tail_relax(m, e, b, a.omega, 0);
    tail_relax(m, e, b, a.omega, 1);
  }
  const LevelMask& cm = a.m[k + 1];
  T* ec = sm + a.off_e[k + 1];
  T* bc = sm + a.off_b[k + 1];
  tail_restrict(m, (const T*)e, (const T*)b, cm, bc, ec, sm + a.off_x);
  int reps = (a.wcycle && k + 1 < a.n - 1) ? 2 : 1;
  for (int q = 0; q < reps; ++q) tail_cycle(a, sm, k + 1);
  tail_prolong(m, e, cm, (const T*)ec);
  for (int s = 0; s < a.post; ++s) {
    tail_relax(m, e, b, a.omega, 0);
    tail_relax(m, e, b, a.omega, 1);
  }
}

template <typename T>
__global__ void __launch_bounds__(kTailThreads) k_gmg_tail(const __grid_constant__ TailArgs<T> a) {
  extern __shared__ __align__(16) unsigned char tail_smem[];
  T* sm = reinterpret_cast<T*>(tail_smem);
  const LevelMask& m0 = a.m[0];
  T* e0 = sm + a.off_e[0];
  T* b0 = sm + a.off_b[0];
  for (int j = threadIdx.y; j < m0.H; j += blockDim.y)
    for (int i = threadIdx.x; i < m0.W; i += blockDim.x) {
      b0[j * m0.W + i] = a.gb[(int64_t)j * a.gld + i];
      e0[j * m0.W + i] = a.zero_init ? (T)0 : a.ge[(int64_t)j * a.gld + i];
    }
  __syncthreads();
  tail_cycle(a, sm, 0);
  for (int j = threadIdx.y; j < m0.H; j += blockDim.y)
    for (int i = threadIdx.x; i < m0.W; i += blockDim.x) a.ge[(int64_t)j * a.gld + i] = e0[j * m0.W + i];
}

// Tiled bc = P^T (b - A e) for analytic (open-box) level pairs: a 32 x 8 block restricts
// a 32 x 8 tile of coarse cells; the fine residual of the tile (18 x 66 cells including
// the window overlap) is computed once into shared memory from e (20 x 68) and b, then
// restricted along x and y.
constexpr int kRX = 32, kRY = 8;
template <typename T>
__global__ void __launch_bounds__(kRX * kRY) k_gmg_residual_restrict_tiled(const T* __restrict__ e,
                                                                            const T* __restrict__ b, int64_t ld,
                                                                            LevelMask fm, T* __restrict__ bc,
                                                                            int64_t ldc, LevelMask cm) {
  constexpr int EW = 2 * kRX + 4, EH = 2 * kRY + 4;  // e tile: fine cols 2I0-2 .. 2I0+2kRX+1
  constexpr int RW = 2 * kRX + 2, RH = 2 * kRY + 2;  // residual tile: fine cols 2I0-1 .. 2I0+2kRX
  __shared__ T se[EH][EW];
  __shared__ T sr[RH][RW];
  __shared__ T sx[RH][kRX];
  const int H = fm.H, W = fm.W, Hc = cm.H, Wc = cm.W;
  const int I0 = blockIdx.x * kRX, J0 = blockIdx.y * kRY;
  const int fj0 = 2 * J0 - 2, fi0 = 2 * I0 - 2;
  const int tid = threadIdx.y * kRX + threadIdx.x;
  for (int q = tid; q < EH * EW; q += kRX * kRY) {
    int r = q / EW, c = q - r * EW;
    int j = fj0 + r, i = fi0 + c;
    se[r][c] = (j >= 0 && j < H && i >= 0 && i < W) ? e[(int64_t)j * ld + i] : (T)0;
  }
  __syncthreads();
  for (int q = tid; q < RH * RW; q += kRX * kRY) {
    int r = q / RW, c = q - r * RW;
    int j = fj0 + 1 + r, i = fi0 + 1 + c;
    T acc = (T)0;
    if (j >= 0 && j < H && i >= 0 && i < W) {
      const T x = se[r + 1][c + 1];
      acc = b[(int64_t)j * ld + i];
      if (i > 0) acc += se[r + 1][c] - x;
      if (i < W - 1) acc += se[r + 1][c + 2] - x;
      if (j > 0) acc += se[r][c + 1] - x;
      if (j < H - 1) acc += se[r + 2][c + 1] - x;
    }
    sr[r][c] = acc;
  }
  __syncthreads();
  const int I = I0 + threadIdx.x;
  for (int r = threadIdx.y; r < RH; r += kRY) {
    T acc = (T)0;
    if (I < Wc) {
#pragma unroll
      for (int d = 0; d < 4; ++d) {
        const int i = 2 * I - 1 + d;
        if (i < 0 || i >= W) continue;
        const T w = (T)w1(i, I, Wc);
        if (w != (T)0) acc += w * sr[r][2 * threadIdx.x + d];
      }
    }
    sx[r][threadIdx.x] = acc;
  }
  __syncthreads();
  const int J = J0 + threadIdx.y;
  if (I >= Wc || J >= Hc) return;
  T acc = (T)0;
#pragma unroll
  for (int d = 0; d < 4; ++d) {
    const int j = 2 * J - 1 + d;
    if (j < 0 || j >= H) continue;
    const T w = (T)w1(j, J, Hc);
    if (w != (T)0) acc += w * sx[2 * threadIdx.y + d][threadIdx.x];
  }
  bc[(int64_t)J * ldc + I] = acc;
}

// ---------------------------------------------------------------- fused tiled level kernels
#include "gmg_tiled.cuh"
#include "gmg_tail_open.cuh"
#include "gmg_regtile.cuh"
#include "gmg_regtile_stage.cuh"

// ---------------------------------------------------------------- plan
struct Level {
  int H = 0, W = 0;
  int64_t ld = 0;              // row stride of the real arrays
  int analytic = 0;            // every cell fluid and every interior face open
  std::vector<uint8_t> code;   // H * W codes (host), empty when analytic
  int fused = 0;               // this level and the next run the fused tiled kernels
  int64_t off_e = 0, off_e2 = 0, off_b = 0, off_code = 0;  // e2: second e buffer (fused levels)
};

}  // namespace sg

struct sg_gmg_plan {
  int H = 0, W = 0, precision = 0, cycle = 0, pre = 0, post = 0, coarsest = 0;
  double omega = 1.0;
  std::vector<sg::Level> levels;
  std::vector<double> pinv;  // coarsest pseudo-inverse, n x n
  // coarsest open-box level above kPinvMaxSide cells a side: exact solve by the cosine
  // transform (k_gmg_coarse_dct) from the tables in dct (C_x, C_y, eigenvalues)
  int coarse_dct = 0;
  int coarse_dct_multi = 0;  // above kDctMaxSide: the four-product form (k_dct_gemm), scratch at off_dct_x
  int coarse_dct_stream = 0;  // ... run as the two streaming launches (k_dct_stream)
  int coarse_dct_cluster = 0;  // ... on clusters of kDcNC CTAs (k_dct_cluster), when they fit
  int64_t dct_cluster_smem[2] = {0, 0};  // forward, inverse
  int dct_fp64 = 0;           // the transform's arithmetic and tables in float64 (FP64 and mixed precision)
  // the first cycle of a graph solve from a zero guess (set while its graph is captured)
  mutable sg::FirstCycle fc{nullptr, 0, 0, 0, 0, 0.0, 0.0};
  // events recorded around the fused fine-level post launches of kernel-by-kernel solves
  // (pairs, consumed in order; sg_gmg_set_post_events)
  mutable std::vector<cudaEvent_t> post_ev;
  mutable size_t post_ev_next = 0;
  int64_t dct_stream_smem = 0;
  int64_t off_dct_x = 0;
  std::vector<double> dct;
  std::vector<float> dct_f;  // the same in float, for FP32 cycles
  int64_t off_dct = 0, dct_smem = 0;
  int tail_start = 0;        // first level handled by the single-block tail kernel
  int tail_open = 0;         // every tail level is an open box (k_gmg_tail_open)
  int64_t tail_smem = 0;     // its dynamic shared memory (bytes)
  int64_t off_pinv = 0, off_bfine = 0, off_partial = 0, off_state = 0, bytes = 0;
  int64_t ld_bfine = 0;
  int64_t n_partial = 0;
  // fused fine level (register tiles): post-smoothing, correction and residual in one
  // kernel; the cycle rhs alternates between levels[0].off_b and off_b2, and off_r64 holds
  // the residual in the precision of p when that differs from the cycle precision
  int fused_ir = 0;
  int64_t off_b2 = 0, off_r64 = 0;
  // cycles per refinement step (classical iterative refinement): with inner >= 2 the body
  // runs `inner` cycles on the cycle-precision correction from zero, then one p += e and one
  // fine-precision residual, instead of the fused fine level's per-cycle correction
  int inner = 1;
  // remove the fluid mean of the rhs before solving (a Neumann problem's rhs must sum to
  // zero; float rounding of a telescoping divergence sum leaves a component no p removes)
  int remove_mean = 0;
  double inv_fluid = 0.0;
  char* ws = nullptr;        // bound device workspace
  // cached solve graph
  cudaStream_t capture_stream = nullptr;
  cudaGraphExec_t exec = nullptr;
  const void* g_p = nullptr;
  const void* g_div = nullptr;
  int64_t g_ldp = 0, g_ldd = 0;
  int g_div_dtype = -1;
  int g_zero = 0;
  int prologue_nodes = 0, body_nodes = 0;
};

namespace sg {

static int64_t align256(int64_t x) { return (x + 255) & ~(int64_t)255; }

static bool level_is_open(const std::vector<uint8_t>& fl, const std::vector<uint8_t>& fu, const std::vector<uint8_t>& fv,
                          int H, int W) {
  for (int j = 0; j < H; ++j)
    for (int i = 0; i < W; ++i)
      if (!fl[(size_t)j * W + i]) return false;
  for (int j = 0; j < H; ++j)
    for (int i = 0; i <= W; ++i) {
      bool want = i >= 1 && i <= W - 1;
      if ((fu[(size_t)j * (W + 1) + i] != 0) != want) return false;
    }
  for (int j = 0; j <= H; ++j)
    for (int i = 0; i < W; ++i) {
      bool want = j >= 1 && j <= H - 1;
      if ((fv[(size_t)j * W + i] != 0) != want) return false;
    }
  return true;
}

static std::vector<uint8_t> pack_codes(const std::vector<uint8_t>& fl, const std::vector<uint8_t>& fu,
                                       const std::vector<uint8_t>& fv, int H, int W) {
  std::vector<uint8_t> c((size_t)H * W);
  for (int j = 0; j < H; ++j)
    for (int i = 0; i < W; ++i) {
      uint8_t x = 0;
      if (fl[(size_t)j * W + i]) x |= C_FLUID;
      if (fu[(size_t)j * (W + 1) + i]) x |= C_L;
      if (fu[(size_t)j * (W + 1) + i + 1]) x |= C_R;
      if (fv[(size_t)j * W + i]) x |= C_D;
      if (fv[(size_t)(j + 1) * W + i]) x |= C_U;
      c[(size_t)j * W + i] = x;
    }
  return c;
}

// Pseudo-inverse of the graph Laplacian A of one level: A+ = (A + Pi)^-1 - Pi, with Pi
// the orthogonal projector onto the constants of each connected fluid component.
static bool coarsest_pinv(const std::vector<uint8_t>& code, int H, int W, std::vector<double>& out) {
  int n = H * W;
  std::vector<double> A((size_t)n * n, 0.0);
  for (int j = 0; j < H; ++j)
    for (int i = 0; i < W; ++i) {
      int k = j * W + i;
      uint8_t c = code[k];
      if (!(c & C_FLUID)) continue;
      int nb[4] = {c & C_L ? k - 1 : -1, c & C_R ? k + 1 : -1, c & C_D ? k - W : -1, c & C_U ? k + W : -1};
      for (int q = 0; q < 4; ++q)
        if (nb[q] >= 0) {
          A[(size_t)k * n + k] += 1.0;
          A[(size_t)k * n + nb[q]] -= 1.0;
        }
    }
  std::vector<int> comp(n, -1);
  std::vector<int> stack;
  std::vector<int> sizes;
  for (int s = 0; s < n; ++s) {
    if (!(code[s] & C_FLUID) || comp[s] >= 0) continue;
    int id = (int)sizes.size();
    sizes.push_back(0);
    stack.push_back(s);
    comp[s] = id;
    while (!stack.empty()) {
      int k = stack.back();
      stack.pop_back();
      sizes[id]++;
      uint8_t c = code[k];
      int nb[4] = {c & C_L ? k - 1 : -1, c & C_R ? k + 1 : -1, c & C_D ? k - W : -1, c & C_U ? k + W : -1};
      for (int q = 0; q < 4; ++q)
        if (nb[q] >= 0 && comp[nb[q]] < 0) {
          comp[nb[q]] = id;
          stack.push_back(nb[q]);
        }
    }
  }
  std::vector<double> M = A;
  for (int a = 0; a < n; ++a)
    for (int b = 0; b < n; ++b)
      if (comp[a] >= 0 && comp[a] == comp[b]) M[(size_t)a * n + b] += 1.0 / sizes[comp[a]];
  for (int a = 0; a < n; ++a)
    if (comp[a] < 0) M[(size_t)a * n + a] = 1.0;  // non-fluid rows: identity, removed below
  std::vector<double> I((size_t)n * n, 0.0);
  for (int a = 0; a < n; ++a) I[(size_t)a * n + a] = 1.0;
  for (int col = 0; col < n; ++col) {  // Gauss-Jordan with partial pivoting
    int piv = col;
    for (int r = col + 1; r < n; ++r)
      if (std::fabs(M[(size_t)r * n + col]) > std::fabs(M[(size_t)piv * n + col])) piv = r;
    if (std::fabs(M[(size_t)piv * n + col]) < 1e-300) return false;
    if (piv != col)
      for (int q = 0; q < n; ++q) {
        std::swap(M[(size_t)piv * n + q], M[(size_t)col * n + q]);
        std::swap(I[(size_t)piv * n + q], I[(size_t)col * n + q]);
      }
    double d = M[(size_t)col * n + col];
    for (int q = 0; q < n; ++q) {
      M[(size_t)col * n + q] /= d;
      I[(size_t)col * n + q] /= d;
    }
    for (int r = 0; r < n; ++r) {
      if (r == col) continue;
      double f = M[(size_t)r * n + col];
      if (f == 0.0) continue;
      for (int q = 0; q < n; ++q) {
        M[(size_t)r * n + q] -= f * M[(size_t)col * n + q];
        I[(size_t)r * n + q] -= f * I[(size_t)col * n + q];
      }
    }
  }
  out.assign((size_t)n * n, 0.0);
  for (int a = 0; a < n; ++a)
    for (int b = 0; b < n; ++b) {
      if (comp[a] < 0 || comp[b] < 0) continue;
      double v = I[(size_t)a * n + b];
      if (comp[a] == comp[b]) v -= 1.0 / sizes[comp[a]];
      out[(size_t)a * n + b] = v;
    }
  return true;
}

// Pseudo-inverse of the open-box operator on an H x W grid (every cell fluid, every
// interior face open); used by the batched solver for its scenes' coarsest levels.
bool open_box_pinv(int H, int W, std::vector<double>& out) {
  std::vector<uint8_t> fl((size_t)H * W, 1), fu((size_t)H * (W + 1), 0), fv((size_t)(H + 1) * W, 0);
  for (int j = 0; j < H; ++j)
    for (int i = 1; i < W; ++i) fu[(size_t)j * (W + 1) + i] = 1;
  for (int j = 1; j < H; ++j)
    for (int i = 0; i < W; ++i) fv[(size_t)j * W + i] = 1;
  return coarsest_pinv(pack_codes(fl, fu, fv, H, W), H, W, out);
}

static LevelMask level_mask(const sg_gmg_plan* p, int k) {
  const Level& L = p->levels[k];
  LevelMask m;
  m.code = L.analytic ? nullptr : (const uint8_t*)(p->ws + L.off_code);
  m.analytic = L.analytic;
  m.H = L.H;
  m.W = L.W;
  return m;
}

template <typename T>
static T* ws_ptr(const sg_gmg_plan* p, int64_t off) {
  return (T*)(p->ws + off);
}

static GmgState* state_ptr(const sg_gmg_plan* p) { return (GmgState*)(p->ws + p->off_state); }

// Shared-memory layout of the open-box tail (elements of T): every level's e planes first
// (zeroed at start), then the b planes, then the restriction and residual scratch.
struct OpenTailLayout {
  int off_e[kMaxLevels], off_b[kMaxLevels], e_total, off_x, off_r, total;
};

static OpenTailLayout open_tail_layout(const std::vector<Level>& levels, int start) {
  OpenTailLayout t;
  std::memset(&t, 0, sizeof(t));
  int n = (int)levels.size() - start;
  int off = 0;
  for (int q = 0; q < n; ++q) {
    const Level& L = levels[start + q];
    const int wh = (L.W + 1) / 2;
    t.off_e[q] = off;
    off += 2 * (L.H + 2) * (wh + 2);
  }
  t.e_total = off;
  for (int q = 0; q < n; ++q) {
    const Level& L = levels[start + q];
    t.off_b[q] = off;
    off += 2 * L.H * ((L.W + 1) / 2);
  }
  t.off_x = off;
  off += levels[start].H * ((levels[start].W + 1) / 2);
  t.off_r = off;
  off += levels[start].H * levels[start].W;
  t.total = off;
  return t;
}

template <typename T>
static int tail_open_launch(const sg_gmg_plan* p, bool zero_init, cudaStream_t s) {
  OpenTailArgs<T> a;
  std::memset(&a, 0, sizeof(a));
  int nl = (int)p->levels.size();
  a.n = nl - p->tail_start;
  OpenTailLayout t = open_tail_layout(p->levels, p->tail_start);
  for (int q = 0; q < a.n; ++q) {
    a.H[q] = p->levels[p->tail_start + q].H;
    a.W[q] = p->levels[p->tail_start + q].W;
    a.off_e[q] = t.off_e[q];
    a.off_b[q] = t.off_b[q];
  }
  a.e_total = t.e_total;
  a.off_x = t.off_x;
  a.off_r = t.off_r;
  const Level& L0 = p->levels[p->tail_start];
  a.ge = ws_ptr<T>(p, L0.off_e);
  a.gb = ws_ptr<T>(p, L0.off_b);
  a.gld = L0.ld;
  a.pinv = (const double*)(p->ws + p->off_pinv);
  a.omega = (T)p->omega;
  a.pre = p->pre;
  a.post = p->post;
  a.wcycle = p->cycle;
  a.zero_init = zero_init ? 1 : 0;
  SG_LAUNCH(k_gmg_tail_open<T><<<1, dim3(32, kOpenTailThreads / 32), p->tail_smem, s>>>(a));
  return SG_OK;
}

template <typename T>
static int tail_launch(const sg_gmg_plan* p, bool zero_init, cudaStream_t s) {
  if (p->tail_open) return tail_open_launch<T>(p, zero_init, s);
  TailArgs<T> a;
  std::memset(&a, 0, sizeof(a));
  int nl = (int)p->levels.size();
  a.n = nl - p->tail_start;
  int64_t off = 0;
  for (int q = 0; q < a.n; ++q) {
    const Level& L = p->levels[p->tail_start + q];
    a.m[q] = level_mask(p, p->tail_start + q);
    a.off_e[q] = (int)off;
    off += (int64_t)L.H * L.W;
    a.off_b[q] = (int)off;
    off += (int64_t)L.H * L.W;
    off = (off + 3) & ~(int64_t)3;
  }
  a.off_x = (int)off;
  const Level& L0 = p->levels[p->tail_start];
  a.ge = ws_ptr<T>(p, L0.off_e);
  a.gb = ws_ptr<T>(p, L0.off_b);
  a.gld = L0.ld;
  a.pinv = (const double*)(p->ws + p->off_pinv);
  a.omega = (T)p->omega;
  a.pre = p->pre;
  a.post = p->post;
  a.wcycle = p->cycle;
  a.zero_init = zero_init ? 1 : 0;
  SG_LAUNCH(k_gmg_tail<T><<<1, dim3(32, kTailThreads / 32), p->tail_smem, s>>>(a));
  return SG_OK;
}

// The fused tiled kernels serve open-box level pairs with 1..3 sweeps per side.
static bool fused_level(const sg_gmg_plan* p, int k) { return p->levels[k].fused != 0; }

// Register tiles on levels of at least SG_GMG_REG_MIN_TILES 64 x 32 blocks, 16 x 16 shared-
// memory tiles below: a small level is latency-bound, and more blocks with less serial work
// each finish sooner. Per V-cycle at 2048^2 (32^2 exact coarsest; mixed / float64 / float32):
// threshold 296 (512^2 on small tiles) 139 / 165 / 125 us, 100 (512^2 on register tiles)
// 137 / 159 / 123, 30 (256^2 too) 141 / 160 / 127, every level 150 / 163 / 136.
#ifndef SG_GMG_REG_MIN_TILES
#define SG_GMG_REG_MIN_TILES 100
#endif
static bool small_tiles(const Level& L) {
  const int64_t large_blocks = (int64_t)((L.W + kTX - 1) / kTX) * ((L.H + kTY - 1) / kTY);
  return large_blocks < SG_GMG_REG_MIN_TILES;
}

// Rows of 32 threads of a shared-memory tile block: kTBY, or SG_TILE_FEW_ROWS on levels of
// at most SG_TILE_FEW_TILES tiles (a wave or less of blocks: more threads per block
// shorten each phase of the block, which is all the level costs).
#ifndef SG_TILE_FEW_TILES
#define SG_TILE_FEW_TILES 256
#endif
#ifndef SG_TILE_FEW_ROWS
#define SG_TILE_FEW_ROWS 16
#endif
static dim3 tile_block(dim3 g) {
  return dim3(kTBX, (int64_t)g.x * g.y <= SG_TILE_FEW_TILES ? SG_TILE_FEW_ROWS : kTBY);
}

template <typename T, int SW, int TX, int TY>
static void launch_pre_t(const sg_gmg_plan* p, int k, bool zero_init, cudaStream_t s) {
  const Level& L = p->levels[k];
  const Level& C = p->levels[k + 1];
  dim3 g((L.W + TX - 1) / TX, (L.H + TY - 1) / TY);
  // reads E0 (nothing for a zero initial guess), writes E1
  SG_LAUNCH(k_gmg_pre_tiled<T, SW, TX, TY><<<g, tile_block(g), PreShape<SW, TX, TY>::template bytes<T>(), s>>>(
      zero_init ? nullptr : ws_ptr<T>(p, L.off_e), ws_ptr<T>(p, L.off_e2), ws_ptr<T>(p, L.off_b), L.ld, L.H, L.W,
      ws_ptr<T>(p, C.off_b), C.ld, C.H, C.W, (T)p->omega));
}

template <typename T, int SW, int TX, int TY>
static void launch_post_t(const sg_gmg_plan* p, int k, cudaStream_t s) {
  const Level& L = p->levels[k];
  const Level& C = p->levels[k + 1];
  dim3 g((L.W + TX - 1) / TX, (L.H + TY - 1) / TY);
  // reads E1 and the coarse correction (the coarse level's E0), writes E0
  SG_LAUNCH(k_gmg_post_tiled<T, SW, TX, TY><<<g, tile_block(g), PostShape<SW, TX, TY>::template bytes<T>(), s>>>(
      ws_ptr<T>(p, L.off_e2), ws_ptr<T>(p, L.off_e), ws_ptr<T>(p, L.off_b), L.ld, L.H, L.W, ws_ptr<T>(p, C.off_e),
      C.ld, C.H, C.W, (T)p->omega));
}

template <typename T, int SW>
static void launch_pre_reg(const sg_gmg_plan* p, int k, bool zero_init, cudaStream_t s, const T* b_alt = nullptr) {
  constexpr int RPT = RegShape<T>::RPT, NW = RegShape<T>::NWARP, MB = RegShape<T>::MINB;
  using S = RegPre<T, SW, RPT, NW>;
  const Level& L = p->levels[k];
  const Level& C = p->levels[k + 1];
  dim3 g((L.W + S::TXO - 1) / S::TXO, (L.H + S::TYO - 1) / S::TYO);
  SG_LAUNCH(k_gmg_pre_reg<T, SW, RPT, NW, MB><<<g, 32 * NW, 0, s>>>(
      zero_init ? nullptr : ws_ptr<T>(p, L.off_e), ws_ptr<T>(p, L.off_e2), ws_ptr<T>(p, L.off_b), b_alt,
      state_ptr(p), L.ld, L.H, L.W, ws_ptr<T>(p, C.off_b), C.ld, C.H, C.W, (T)p->omega));
}

template <typename T, int SW>
static void launch_post_reg(const sg_gmg_plan* p, int k, cudaStream_t s) {
  constexpr int RPT = RegShape<T>::RPT, NW = RegShape<T>::NWARP, MB = RegShape<T>::MINB;
  using S = RegPost<T, SW, RPT, NW>;
  const Level& L = p->levels[k];
  const Level& C = p->levels[k + 1];
  dim3 g((L.W + S::TXO - 1) / S::TXO, (L.H + S::TYO - 1) / S::TYO);
  SG_LAUNCH(k_gmg_post_reg<T, SW, RPT, NW, MB><<<g, 32 * NW, 0, s>>>(
      ws_ptr<T>(p, L.off_e2), ws_ptr<T>(p, L.off_e), ws_ptr<T>(p, L.off_b), L.ld, L.H, L.W, ws_ptr<T>(p, C.off_e),
      C.ld, C.H, C.W, (T)p->omega));
}

// Grid of the fused fine-level post kernel (also the number of its partial sums).
template <typename TC>
static dim3 post_final_grid(const sg_gmg_plan* p) {
  constexpr int RPT = RegShape<TC>::RPT_FINAL, NW = RegShape<TC>::NWARP_FINAL;
  const int sw = p->post < 1 ? 1 : (p->post > 3 ? 3 : p->post);
  const int halo = 2 * sw + 2, txo = kRW - 2 * halo, tyo = NW * RPT - 2 * halo;
  const Level& L = p->levels[0];
  return dim3((L.W + txo - 1) / txo, (L.H + tyo - 1) / tyo);
}

template <typename TC, typename TP, int SW>
static void launch_post_final(const sg_gmg_plan* p, TP* pp, int64_t ldp, cudaStream_t s) {
  constexpr int RPT = RegShape<TC>::RPT_FINAL, NW = RegShape<TC>::NWARP_FINAL, MB = RegShape<TC>::MINB_FINAL;
  const Level& L = p->levels[0];
  const Level& C = p->levels[1];
  TP* r64 = p->off_r64 ? (TP*)(p->ws + p->off_r64) : nullptr;
  // p and r64 staged in shared memory by bulk copies when every owned row of theirs starts on
  // a 16-byte boundary (the workspace rows always do; the caller's p must)
  const bool staged = ((uintptr_t)pp % 16) == 0 && ((size_t)ldp * sizeof(TP)) % 16 == 0 &&
                      ((uintptr_t)p->ws % 16) == 0 && ((size_t)L.ld * sizeof(TP)) % 16 == 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  if (p->post_ev_next + 1 < p->post_ev.size()) {  // timing events, outside stream capture only
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusActive;
    if (cudaStreamIsCapturing(s, &cs) == cudaSuccess && cs == cudaStreamCaptureStatusNone) {
      ev0 = p->post_ev[p->post_ev_next];
      ev1 = p->post_ev[p->post_ev_next + 1];
      p->post_ev_next += 2;
    }
  }
  if (ev0) cudaEventRecord(ev0, s);
  if (staged) {
    SG_LAUNCH(k_gmg_post_final_stage<TC, TP, SW, RPT, NW, MB><<<post_final_grid<TC>(p), 32 * NW, 0, s>>>(
        ws_ptr<TC>(p, L.off_e2), ws_ptr<TC>(p, L.off_b), ws_ptr<TC>(p, p->off_b2), state_ptr(p), L.ld, L.H, L.W,
        ws_ptr<TC>(p, C.off_e), C.ld, C.H, C.W, (TC)p->omega, pp, ldp, r64, (double*)(p->ws + p->off_partial),
        p->fc));
  } else {
    SG_LAUNCH(k_gmg_post_final_reg<TC, TP, SW, RPT, NW, MB><<<post_final_grid<TC>(p), 32 * NW, 0, s>>>(
        ws_ptr<TC>(p, L.off_e2), ws_ptr<TC>(p, L.off_b), ws_ptr<TC>(p, p->off_b2), state_ptr(p), L.ld, L.H, L.W,
        ws_ptr<TC>(p, C.off_e), C.ld, C.H, C.W, (TC)p->omega, pp, ldp, r64, (double*)(p->ws + p->off_partial),
        p->fc));
  }
  if (ev1) cudaEventRecord(ev1, s);
}

// Large levels: register tiles; small levels: 16 x 16 shared-memory tiles.
template <typename T, int SW>
static void launch_pre(const sg_gmg_plan* p, int k, bool zero_init, cudaStream_t s) {
  if (small_tiles(p->levels[k]))
    launch_pre_t<T, SW, kSX, kSY>(p, k, zero_init, s);
  else
    launch_pre_reg<T, SW>(p, k, zero_init, s);
}

template <typename T, int SW>
static void launch_post(const sg_gmg_plan* p, int k, cudaStream_t s) {
  if (small_tiles(p->levels[k]))
    launch_post_t<T, SW, kSX, kSY>(p, k, s);
  else
    launch_post_reg<T, SW>(p, k, s);
}

template <typename T>
static int set_tiled_smem_limits() {
  cudaError_t e = cudaSuccess;
#define SG_TILED_ATTR(SW, TX, TY)                                                                                  \
  e = cudaFuncSetAttribute(k_gmg_pre_tiled<T, SW, TX, TY>, cudaFuncAttributeMaxDynamicSharedMemorySize,            \
                           (int)PreShape<SW, TX, TY>::template bytes<T>());                                        \
  if (e != cudaSuccess) return fail(SG_ERR_CUDA, "smem attr: %s", cudaGetErrorString(e));                          \
  e = cudaFuncSetAttribute(k_gmg_post_tiled<T, SW, TX, TY>, cudaFuncAttributeMaxDynamicSharedMemorySize,           \
                           (int)PostShape<SW, TX, TY>::template bytes<T>());                                       \
  if (e != cudaSuccess) return fail(SG_ERR_CUDA, "smem attr: %s", cudaGetErrorString(e));
  SG_TILED_ATTR(1, kTX, kTY)
  SG_TILED_ATTR(2, kTX, kTY)
  SG_TILED_ATTR(3, kTX, kTY)
  SG_TILED_ATTR(1, kSX, kSY)
  SG_TILED_ATTR(2, kSX, kSY)
  SG_TILED_ATTR(3, kSX, kSY)
#undef SG_TILED_ATTR
  return SG_OK;
}

// Thread groups of k_dct_stream for a level W cells wide (at most 256 threads a block).
static int dct_stream_groups(int W) {
  const int cw = (W + 31) / 32 * 32;
  return cw <= 64 ? 4 : (cw <= 128 ? 2 : 1);
}

// The streaming form of the coarsest cosine transform applies when every streamed row (of B,
// the tables and the scratch) starts and ends on 16-byte boundaries and its shared memory
// fits one block; otherwise the four-product form stays. T: level type, TA: arithmetic type.
// The workspace itself is 256-byte aligned (sg_gmg_bind checks it).
template <typename T, typename TA>
static bool dct_stream_fits(const Level& C) {
  return ((size_t)C.W * sizeof(T)) % 16 == 0 && ((size_t)C.W * sizeof(TA)) % 16 == 0 &&
         ((size_t)C.ld * sizeof(T)) % 16 == 0 && dct_stream_layout<TA>(C.H, C.W).bytes <= (size_t)kDsSmemBudget;
}

template <typename T, typename TA>
static int set_dct_stream_smem(const sg_gmg_plan* p) {
  const int bytes = (int)p->dct_stream_smem;
  cudaError_t e = cudaSuccess;
#define SG_DS_ATTR(NKG)                                                                                            \
  if (e == cudaSuccess)                                                                                            \
    e = cudaFuncSetAttribute(k_dct_stream<T, TA, NKG, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes); \
  if (e == cudaSuccess)                                                                                            \
    e = cudaFuncSetAttribute(k_dct_stream<T, TA, NKG, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  switch (dct_stream_groups(p->levels.back().W)) {
    case 4: SG_DS_ATTR(4) break;
    case 2: SG_DS_ATTR(2) break;
    default: SG_DS_ATTR(1) break;
  }
#undef SG_DS_ATTR
  if (e == cudaSuccess && p->coarse_dct_cluster) {
    const int bf = (int)p->dct_cluster_smem[0], bi = (int)p->dct_cluster_smem[1];
#define SG_DC_ATTR(NKG)                                                                                            \
  if (e == cudaSuccess)                                                                                            \
    e = cudaFuncSetAttribute(k_dct_cluster<T, TA, NKG, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, bf);   \
  if (e == cudaSuccess)                                                                                            \
    e = cudaFuncSetAttribute(k_dct_cluster<T, TA, NKG, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, bi);
    switch (dct_stream_groups(p->levels.back().W)) {
      case 4: SG_DC_ATTR(4) break;
      case 2: SG_DC_ATTR(2) break;
      default: SG_DC_ATTR(1) break;
    }
#undef SG_DC_ATTR
  }
  return e == cudaSuccess ? SG_OK : fail(SG_ERR_CUDA, "cosine-transform stream smem: %s", cudaGetErrorString(e));
}

template <typename T, typename TA, int NKG>
static void dct_stream_launch_g(const sg_gmg_plan* p, const Level& C, cudaStream_t s) {
  const TA* tab = (const TA*)(p->ws + p->off_dct);
  TA* X = (TA*)(p->ws + p->off_dct_x);
  const int cw = (C.W + 31) / 32 * 32;
  if (p->coarse_dct_cluster) {
    const dim3 gc((unsigned)(((C.H + kDsRB - 1) / kDsRB) * kDcNC)), bc(cw * NKG);
    SG_LAUNCH((k_dct_cluster<T, TA, NKG, false><<<gc, bc, (size_t)p->dct_cluster_smem[0], s>>>(
        C.H, C.W, ws_ptr<T>(p, C.off_b), C.ld, tab, X, nullptr, 0, state_ptr(p))));
    SG_LAUNCH((k_dct_cluster<T, TA, NKG, true><<<gc, bc, (size_t)p->dct_cluster_smem[1], s>>>(
        C.H, C.W, nullptr, 0, tab, X, ws_ptr<T>(p, C.off_e), C.ld, state_ptr(p))));
    return;
  }
  const dim3 g((C.H + kDsRB - 1) / kDsRB), b(cw * NKG);
  const size_t sm = (size_t)p->dct_stream_smem;
  SG_LAUNCH((k_dct_stream<T, TA, NKG, false><<<g, b, sm, s>>>(C.H, C.W, ws_ptr<T>(p, C.off_b), C.ld, tab, X, nullptr,
                                                              0, state_ptr(p))));
  SG_LAUNCH((k_dct_stream<T, TA, NKG, true><<<g, b, sm, s>>>(C.H, C.W, nullptr, 0, tab, X, ws_ptr<T>(p, C.off_e),
                                                             C.ld, state_ptr(p))));
}

template <typename T, typename TA>
static void dct_stream_launch(const sg_gmg_plan* p, const Level& C, cudaStream_t s) {
  switch (dct_stream_groups(C.W)) {
    case 4: dct_stream_launch_g<T, TA, 4>(p, C, s); break;
    case 2: dct_stream_launch_g<T, TA, 2>(p, C, s); break;
    default: dct_stream_launch_g<T, TA, 1>(p, C, s); break;
  }
}

// One cycle on level k for A_k e_k = b_k; zero_init: start from e_k = 0.
template <typename T>
static void cycle(const sg_gmg_plan* p, int k, bool zero_init, cudaStream_t s) {
  if (p->coarse_dct && k == (int)p->levels.size() - 1) {
    const Level& C = p->levels[k];
    if (p->coarse_dct_stream) {
      if (p->dct_fp64)
        dct_stream_launch<T, double>(p, C, s);
      else
        dct_stream_launch<T, T>(p, C, s);
      return;
    }
    if (p->coarse_dct_multi) {
      const int H = C.H, W = C.W;
      const T* tab = ws_ptr<T>(p, p->off_dct);
      const T* cx = tab;                          // cx[k W + i]
      const T* cy = tab + 2 * (int64_t)W * W;      // cy[m H + j]
      const T* lx = cy + (int64_t)H * H;
      const T* ly = lx + W;
      T* X = ws_ptr<T>(p, p->off_dct_x);
      T* Y = X + (int64_t)H * W;
      const dim3 g((W + kDT - 1) / kDT, (H + kDT - 1) / kDT);
      const size_t sw = dct_gemm_smem<T>(W), sh = dct_gemm_smem<T>(H);
      SG_LAUNCH((k_dct_gemm<T, false, true, 0><<<g, kDT * kDT, sw, s>>>(H, W, W, ws_ptr<T>(p, C.off_b), C.ld, cx, W,
                                                                         X, W, nullptr, nullptr)));
      SG_LAUNCH((k_dct_gemm<T, false, false, 1><<<g, kDT * kDT, sh, s>>>(H, W, H, cy, H, X, W, Y, W, ly, lx)));
      SG_LAUNCH((k_dct_gemm<T, true, false, 0><<<g, kDT * kDT, sh, s>>>(H, W, H, cy, H, Y, W, X, W, nullptr,
                                                                         nullptr)));
      SG_LAUNCH((k_dct_gemm<T, false, false, 0><<<g, kDT * kDT, sw, s>>>(H, W, W, X, W, cx, W,
                                                                          ws_ptr<T>(p, C.off_e), C.ld, nullptr,
                                                                          nullptr)));
      return;
    }
    if (p->dct_fp64)
      SG_LAUNCH((k_gmg_coarse_dct<T, double><<<1, 1024, p->dct_smem, s>>>(
          ws_ptr<T>(p, C.off_b), C.ld, ws_ptr<T>(p, C.off_e), C.ld, C.H, C.W, (const double*)(p->ws + p->off_dct))));
    else
      SG_LAUNCH((k_gmg_coarse_dct<T, T><<<1, 1024, p->dct_smem, s>>>(ws_ptr<T>(p, C.off_b), C.ld, ws_ptr<T>(p, C.off_e),
                                                                      C.ld, C.H, C.W, ws_ptr<T>(p, p->off_dct))));
    return;
  }
  if (k == p->tail_start) {
    tail_launch<T>(p, zero_init, s);
    return;
  }
  const int nl = (int)p->levels.size();
  if (fused_level(p, k)) {
    switch (p->pre) {
      case 1: launch_pre<T, 1>(p, k, zero_init, s); break;
      case 2: launch_pre<T, 2>(p, k, zero_init, s); break;
      default: launch_pre<T, 3>(p, k, zero_init, s); break;
    }
    int reps = (p->cycle == 1 && k + 1 < nl - 1) ? 2 : 1;
    for (int q = 0; q < reps; ++q) cycle<T>(p, k + 1, q == 0, s);
    switch (p->post) {
      case 1: launch_post<T, 1>(p, k, s); break;
      case 2: launch_post<T, 2>(p, k, s); break;
      default: launch_post<T, 3>(p, k, s); break;
    }
    return;
  }
  const Level& L = p->levels[k];
  LevelMask m = level_mask(p, k);
  T* e = ws_ptr<T>(p, L.off_e);
  T* b = ws_ptr<T>(p, L.off_b);
  const Level& C = p->levels[k + 1];
  LevelMask cm = level_mask(p, k + 1);
  dim3 gh = grid2d((L.W + 1) / 2, L.H);
  if (zero_init && p->pre == 0) cudaMemsetAsync(e, 0, sizeof(T) * L.ld * L.H, s);
  for (int sw = 0; sw < p->pre; ++sw)
    for (int color = 0; color < 2; ++color)
      SG_LAUNCH(k_gmg_rbgs<T><<<gh, block2d(), 0, s>>>(L.H, L.W, e, L.ld, b, m, (T)p->omega, color,
                                                         (zero_init && sw == 0 && color == 0) ? 1 : 0));
  if (L.analytic && C.analytic)
    SG_LAUNCH(k_gmg_residual_restrict_tiled<T><<<dim3((C.W + kRX - 1) / kRX, (C.H + kRY - 1) / kRY), dim3(kRX, kRY),
                                                 0, s>>>(e, b, L.ld, m, ws_ptr<T>(p, C.off_b), C.ld, cm));
  else
    SG_LAUNCH(k_gmg_residual_restrict<T><<<grid2d(C.W, C.H), block2d(), 0, s>>>(e, b, L.ld, m, ws_ptr<T>(p, C.off_b),
                                                                                 C.ld, cm));
  int reps = (p->cycle == 1 && k + 1 < nl - 1) ? 2 : 1;
  for (int q = 0; q < reps; ++q) cycle<T>(p, k + 1, q == 0, s);
  SG_LAUNCH(k_gmg_prolong_add<T><<<grid2d(L.W, L.H), block2d(), 0, s>>>(ws_ptr<T>(p, C.off_e), C.ld, cm, e, L.ld, m));
  for (int sw = 0; sw < p->post; ++sw)
    for (int color = 0; color < 2; ++color)
      SG_LAUNCH(k_gmg_rbgs<T><<<gh, block2d(), 0, s>>>(L.H, L.W, e, L.ld, b, m, (T)p->omega, color, 0));
}

// Prologue: bf = alpha div, ||bf||, r0 = bf - A p -> cycle rhs, relres0 and the loop condition.
// zero_guess: p is not read; it starts at 0 (written here), so the first residual is bf.
template <typename TP, typename TD, typename TC>
static void prologue(const sg_gmg_plan* p, TP* pp, int64_t ldp, const TD* div, int64_t ldd,
                     cudaGraphConditionalHandle h, int use_handle, cudaStream_t s, bool zero_guess = false) {
  const Level& L = p->levels[0];
  LevelMask m = level_mask(p, 0);
  double* part = (double*)(p->ws + p->off_partial);
  GmgState* st = state_ptr(p);
  dim3 g = grid_wide(L.W, L.H);
  TP* bf = (TP*)(p->ws + p->off_bfine);
  TP* r64 = p->off_r64 ? (TP*)(p->ws + p->off_r64) : nullptr;
  if (p->remove_mean) {
    SG_LAUNCH(k_gmg_rhs_sum<TD><<<g, block2d(), 0, s>>>(L.H, L.W, div, ldd, m, part));
    SG_LAUNCH(k_gmg_finalize_mean<<<1, 1024, 0, s>>>(part, (int)(g.x * g.y), st, p->inv_fluid));
  }
  // from a zero guess the fused fine level carries the residual from here on (b0 / r64), so
  // the FP64 rhs itself is not kept
  TP* bkeep = (zero_guess && p->fused_ir && p->inner <= 1) ? nullptr : bf;
  // the first cycle of such a solve forms r64 from the divergence itself (FirstCycle), so the
  // prologue does not write it
  SG_LAUNCH(k_gmg_rhs<TD, TP, TC><<<g, block2d(), 0, s>>>(L.H, L.W, div, ldd, st, m, bkeep, p->ld_bfine, part,
                                                          zero_guess ? pp : nullptr, ldp, ws_ptr<TC>(p, L.off_b), L.ld,
                                                          (zero_guess && p->fc.active) ? nullptr : r64,
                                                          p->remove_mean));
  SG_LAUNCH(k_gmg_finalize_norm<<<1, 1024, 0, s>>>(part, (int)(g.x * g.y), st));
  if (zero_guess) {
    SG_LAUNCH(k_gmg_finalize_rel<<<1, 1024, 0, s>>>(part, (int)(g.x * g.y), st, h, use_handle, 0));
    return;
  }
  SG_LAUNCH(k_gmg_fine_residual<TP, TC><<<g, block2d(), 0, s>>>(L.H, L.W, pp, ldp, bf, p->ld_bfine, m,
                                                                   ws_ptr<TC>(p, L.off_b), L.ld,
                                                                   r64, part));
  SG_LAUNCH(k_gmg_finalize_rel<<<1, 1024, 0, s>>>(part, (int)(g.x * g.y), st, h, use_handle, 0));
}

// Body: one cycle, p += e, new residual, relres and the loop condition.
template <typename TP, typename TC>
static void body(const sg_gmg_plan* p, TP* pp, int64_t ldp, cudaGraphConditionalHandle h, int use_handle,
                 cudaStream_t s) {
  const Level& L = p->levels[0];
  LevelMask m = level_mask(p, 0);
  double* part = (double*)(p->ws + p->off_partial);
  GmgState* st = state_ptr(p);
  if (p->fused_ir && p->inner <= 1) {
    // pre (rhs by cycle parity) -> coarse levels -> post + correction + next residual
    const TC* b_alt = ws_ptr<TC>(p, p->off_b2);
    switch (p->pre) {
      case 1: launch_pre_reg<TC, 1>(p, 0, true, s, b_alt); break;
      case 2: launch_pre_reg<TC, 2>(p, 0, true, s, b_alt); break;
      default: launch_pre_reg<TC, 3>(p, 0, true, s, b_alt); break;
    }
    const int nl = (int)p->levels.size();
    int reps = (p->cycle == 1 && 1 < nl - 1) ? 2 : 1;
    for (int q = 0; q < reps; ++q) cycle<TC>(p, 1, q == 0, s);
    switch (p->post) {
      case 1: launch_post_final<TC, TP, 1>(p, pp, ldp, s); break;
      case 2: launch_post_final<TC, TP, 2>(p, pp, ldp, s); break;
      default: launch_post_final<TC, TP, 3>(p, pp, ldp, s); break;
    }
    dim3 gf = post_final_grid<TC>(p);
    SG_LAUNCH(k_gmg_finalize_rel<<<1, 1024, 0, s>>>(part, (int)(gf.x * gf.y), st, h, use_handle, 1));
    return;
  }
  dim3 g = grid_wide(L.W, L.H);
  const int inner = p->inner < 1 ? 1 : p->inner;
  for (int q = 0; q < inner; ++q) cycle<TC>(p, 0, q == 0, s);
  SG_LAUNCH(k_gmg_correct<TP, TC><<<g, block2d(), 0, s>>>(L.H, L.W, pp, ldp, ws_ptr<TC>(p, L.off_e), L.ld));
  SG_LAUNCH(k_gmg_fine_residual<TP, TC><<<g, block2d(), 0, s>>>(L.H, L.W, pp, ldp, (const TP*)(p->ws + p->off_bfine),
                                                                   p->ld_bfine, m, ws_ptr<TC>(p, L.off_b), L.ld,
                                                                   (TP*)nullptr, part));
  SG_LAUNCH(k_gmg_finalize_rel<<<1, 1024, 0, s>>>(part, (int)(g.x * g.y), st, h, use_handle, inner));
}

static unsigned long long counter() { return launch_count(); }

#define SG_CUDA_TRY(x, what)                                                              \
  do {                                                                                    \
    cudaError_t _e = (x);                                                                 \
    if (_e != cudaSuccess) return fail(SG_ERR_CUDA, "%s: %s", what, cudaGetErrorString(_e)); \
  } while (0)

// Capture prologue + WHILE(body) into one executable graph for these pointers.
template <typename TP, typename TD, typename TC>
static int build_graph(sg_gmg_plan* p, TP* pp, int64_t ldp, const TD* div, int64_t ldd, bool zero_guess) {
  if (p->exec) {
    cudaGraphExecDestroy(p->exec);
    p->exec = nullptr;
  }
  if (!p->capture_stream) SG_CUDA_TRY(cudaStreamCreateWithFlags(&p->capture_stream, cudaStreamNonBlocking), "stream");
  cudaStream_t cs = p->capture_stream;
  cudaGraph_t g = nullptr;
  SG_CUDA_TRY(cudaGraphCreate(&g, 0), "cudaGraphCreate");
  cudaGraphConditionalHandle h;
  SG_CUDA_TRY(cudaGraphConditionalHandleCreate(&h, g, 0, 0), "cudaGraphConditionalHandleCreate");
  // a zero-guess solve on the fused fine level starts from p = 0 and r64 = alpha div: its first
  // post kernel forms both itself when the divergence rows can be staged (16-byte units)
  struct FcGuard {
    const sg_gmg_plan* p;
    ~FcGuard() { p->fc = FirstCycle{nullptr, 0, 0, 0, 0, 0.0, 0.0}; }
  } fc_guard{p};
  const bool fc_ok = zero_guess && p->fused_ir && p->inner <= 1 && ((uintptr_t)div % 16) == 0 &&
                     ((size_t)ldd * sizeof(TD)) % 16 == 0;
  p->fc = FirstCycle{fc_ok ? (const void*)div : nullptr, ldd, sizeof(TD) == 8 ? 1 : 0, p->remove_mean ? 1 : 0,
                     fc_ok ? 1 : 0, 0.0, 0.0};
  SG_CUDA_TRY(cudaStreamBeginCaptureToGraph(cs, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal),
              "begin capture");
  unsigned long long c0 = counter();
  prologue<TP, TD, TC>(p, pp, ldp, div, ldd, h, 1, cs, zero_guess);
  unsigned long long c1 = counter();
  cudaStreamCaptureStatus cst;
  cudaGraph_t cg = nullptr;
  const cudaGraphNode_t* deps = nullptr;
  size_t ndeps = 0;
  SG_CUDA_TRY(cudaStreamGetCaptureInfo(cs, &cst, nullptr, &cg, &deps, &ndeps), "capture info");
  alignas(cudaGraphNodeParams) unsigned char cpbuf[sizeof(cudaGraphNodeParams)];
  std::memset(cpbuf, 0, sizeof(cpbuf));
  cudaGraphNodeParams& cp = *reinterpret_cast<cudaGraphNodeParams*>(cpbuf);
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t cnode;
  SG_CUDA_TRY(cudaGraphAddNode(&cnode, cg, deps, ndeps, &cp), "add conditional node");
  cudaGraph_t bodyg = cp.conditional.phGraph_out[0];
  SG_CUDA_TRY(cudaStreamUpdateCaptureDependencies(cs, &cnode, 1, cudaStreamSetCaptureDependencies), "update deps");
  SG_CUDA_TRY(cudaStreamEndCapture(cs, &g), "end capture");
  SG_CUDA_TRY(cudaStreamBeginCaptureToGraph(cs, bodyg, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal),
              "begin body capture");
  body<TP, TC>(p, pp, ldp, h, 1, cs);
  unsigned long long c2 = counter();
  SG_CUDA_TRY(cudaStreamEndCapture(cs, &bodyg), "end body capture");
  cudaError_t e = cudaGraphInstantiate(&p->exec, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return fail(SG_ERR_CUDA, "cudaGraphInstantiate: %s", cudaGetErrorString(e));
  p->prologue_nodes = (int)(c1 - c0);
  p->body_nodes = (int)(c2 - c1);
  p->g_p = pp;
  p->g_ldp = ldp;
  p->g_div = div;
  p->g_ldd = ldd;
  p->g_div_dtype = sizeof(TD) == 4 ? SG_F32 : SG_F64;
  p->g_zero = zero_guess ? 1 : 0;
  return SG_OK;
}

template <typename TP, typename TD, typename TC>
static int solve_async_impl(sg_gmg_plan* p, TP* pp, int64_t ldp, const TD* div, int64_t ldd, double alpha, double tol,
                            int max_cycles, cudaStream_t s, bool zero_guess) {
  int dd = sizeof(TD) == 4 ? SG_F32 : SG_F64;
  if (!p->exec || p->g_p != pp || p->g_ldp != ldp || p->g_div != div || p->g_ldd != ldd || p->g_div_dtype != dd ||
      p->g_zero != (zero_guess ? 1 : 0)) {
    int rc = build_graph<TP, TD, TC>(p, pp, ldp, div, ldd, zero_guess);
    if (rc != SG_OK) return rc;
  }
  SG_LAUNCH(k_gmg_set_params<<<1, 1, 0, s>>>(state_ptr(p), alpha, tol, max_cycles));
  SG_CUDA_TRY(cudaGraphLaunch(p->exec, s), "cudaGraphLaunch");
  return check_launch("sg_gmg_solve_async");
}

// Eager (non-graph) execution of exactly n cycles; capturable by the caller.
template <typename TP, typename TD, typename TC>
static int cycles_eager_impl(sg_gmg_plan* p, TP* pp, int64_t ldp, const TD* div, int64_t ldd, double alpha, int n,
                             double* relres_dev, cudaStream_t s) {
  SG_LAUNCH(k_gmg_set_params<<<1, 1, 0, s>>>(state_ptr(p), alpha, -1.0, n));
  cudaGraphConditionalHandle none = 0;
  prologue<TP, TD, TC>(p, pp, ldp, div, ldd, none, 0, s);
  for (int c = 0; c < n; ++c) body<TP, TC>(p, pp, ldp, none, 0, s);
  int m = std::min(n + 1, kHist);
  SG_CUDA_TRY(cudaMemcpyAsync(relres_dev, state_ptr(p)->history, sizeof(double) * m, cudaMemcpyDeviceToDevice, s),
              "history copy");
  return check_launch("sg_gmg_cycles_async");
}

template <typename TP, typename TD, typename TC>
static int solve_async_typed(sg_gmg_plan* plan, void* p, int64_t ld_p, const void* div, int64_t ld_div, double alpha,
                             double tol, int max_cycles, cudaStream_t s, bool zero_guess) {
  return solve_async_impl<TP, TD, TC>(plan, (TP*)p, ld_p, (const TD*)div, ld_div, alpha, tol, max_cycles, s,
                                      zero_guess);
}

template <typename TP, typename TD, typename TC>
static int cycles_typed(sg_gmg_plan* plan, void* p, int64_t ld_p, const void* div, int64_t ld_div, double alpha, int n,
                        double* relres_dev, cudaStream_t s) {
  return cycles_eager_impl<TP, TD, TC>(plan, (TP*)p, ld_p, (const TD*)div, ld_div, alpha, n, relres_dev, s);
}

}  // namespace sg

using namespace sg;

extern "C" {

int sg_gmg_plan_create(sg_gmg_plan** out, int64_t H, int64_t W, int mask_mode, const uint8_t* is_fluid,
                       const uint8_t* fmu, const uint8_t* fmv, int coarsest, double omega, int pre_sweeps,
                       int post_sweeps, int cycle_type, int precision) {
  SG_REQUIRE(out, "null plan pointer");
  *out = nullptr;
  SG_REQUIRE(H >= 1 && W >= 1 && H <= (1 << 16) && W <= (1 << 16), "bad grid %lld x %lld", (long long)H, (long long)W);
  SG_REQUIRE(coarsest >= 1 && coarsest <= kDctMultiMaxSide, "coarsest must be in 1..%d", kDctMultiMaxSide);
  SG_REQUIRE(omega > 0.0 && omega < 2.0, "omega must be in (0, 2)");
  SG_REQUIRE(pre_sweeps >= 0 && post_sweeps >= 0 && pre_sweeps + post_sweeps >= 1, "need at least one smoothing sweep");
  SG_REQUIRE(pre_sweeps <= 16 && post_sweeps <= 16, "at most 16 sweeps per side");
  SG_REQUIRE(cycle_type == 0 || cycle_type == 1, "cycle must be 0 (V) or 1 (W)");
  SG_REQUIRE(precision >= SG_GMG_FP32 && precision <= SG_GMG_MIXED, "bad precision");
  std::vector<uint8_t> fl((size_t)H * W), fu((size_t)H * (W + 1), 0), fv((size_t)(H + 1) * W, 0);
  if (mask_mode == SG_MASK_PLANES) {
    SG_REQUIRE(is_fluid && fmu && fmv, "host mask planes required");
    std::memcpy(fl.data(), is_fluid, fl.size());
    std::memcpy(fu.data(), fmu, fu.size());
    std::memcpy(fv.data(), fmv, fv.size());
  } else if (mask_mode == SG_MASK_OPEN || mask_mode == SG_MASK_RING) {
    bool ring = mask_mode == SG_MASK_RING;
    for (int64_t j = 0; j < H; ++j)
      for (int64_t i = 0; i <= W; ++i)
        fu[(size_t)j * (W + 1) + i] = ring ? (j >= 1 && j <= H - 2 && i >= 2 && i <= W - 2) : (i >= 1 && i <= W - 1);
    for (int64_t j = 0; j <= H; ++j)
      for (int64_t i = 0; i < W; ++i)
        fv[(size_t)j * W + i] = ring ? (i >= 1 && i <= W - 2 && j >= 2 && j <= H - 2) : (j >= 1 && j <= H - 1);
    for (int64_t j = 0; j < H; ++j)
      for (int64_t i = 0; i < W; ++i)
        fl[(size_t)j * W + i] = fu[(size_t)j * (W + 1) + i] || fu[(size_t)j * (W + 1) + i + 1] ||
                                fv[(size_t)j * W + i] || fv[(size_t)(j + 1) * W + i];
  } else {
    return fail(SG_ERR_ARG, "bad mask mode %d", mask_mode);
  }
  sg_gmg_plan* p = new sg_gmg_plan();
  p->H = (int)H;
  p->W = (int)W;
  p->precision = precision;
  p->cycle = cycle_type;
  p->pre = pre_sweeps;
  p->post = post_sweeps;
  p->coarsest = coarsest;
  p->omega = omega;
  {
    int64_t nf = 0;
    for (uint8_t f : fl) nf += f ? 1 : 0;
    p->inv_fluid = nf > 0 ? 1.0 / (double)nf : 0.0;
  }
  int h = (int)H, w = (int)W;
  while (true) {
    Level L;
    L.H = h;
    L.W = w;
    L.analytic = level_is_open(fl, fu, fv, h, w) ? 1 : 0;
    if (!L.analytic) L.code = pack_codes(fl, fu, fv, h, w);
    p->levels.push_back(L);
    if (std::max(h, w) <= coarsest || (int)p->levels.size() == kMaxLevels) break;
    int hc = (h + 1) / 2, wc = (w + 1) / 2;
    std::vector<uint8_t> cfl((size_t)hc * wc, 0), cfu((size_t)hc * (wc + 1), 0), cfv((size_t)(hc + 1) * wc, 0);
    for (int J = 0; J < hc; ++J)
      for (int I = 0; I < wc; ++I) {
        bool any = false;
        for (int dj = 0; dj < 2; ++dj)
          for (int di = 0; di < 2; ++di) {
            int jj = 2 * J + dj, ii = 2 * I + di;
            if (jj < h && ii < w && fl[(size_t)jj * w + ii]) any = true;
          }
        cfl[(size_t)J * wc + I] = any;
      }
    for (int J = 0; J < hc; ++J)
      for (int I = 1; I < wc; ++I) cfu[(size_t)J * (wc + 1) + I] = cfl[(size_t)J * wc + I - 1] && cfl[(size_t)J * wc + I];
    for (int J = 1; J < hc; ++J)
      for (int I = 0; I < wc; ++I) cfv[(size_t)J * wc + I] = cfl[(size_t)(J - 1) * wc + I] && cfl[(size_t)J * wc + I];
    fl.swap(cfl);
    fu.swap(cfu);
    fv.swap(cfv);
    h = hc;
    w = wc;
  }
  if (std::max(p->levels.back().H, p->levels.back().W) > coarsest) {
    delete p;
    return fail(SG_ERR_CAPACITY, "grid needs more than %d levels", kMaxLevels);
  }
  Level& last = p->levels.back();
  if (std::max(last.H, last.W) > kPinvMaxSide) {
    // above the dense pseudo-inverse's size: the cosine transform, which needs an open box
    if (!last.analytic) {
      delete p;
      return fail(SG_ERR_ARG, "a coarsest level above %d cells a side must be an open box (no obstacles); "
                  "lower coarsest", kPinvMaxSide);
    }
    p->coarse_dct = 1;
    p->coarse_dct_multi = std::max(last.H, last.W) > kDctMaxSide ? 1 : 0;
    if (p->coarse_dct_multi && last.H % kDcNC == 0 && last.W % kDcNC == 0)
      coarse_dct_tables_split(last.H, last.W, kDcNC, p->dct);  // + C_x^T split for k_dct_cluster
    else
      coarse_dct_tables(last.H, last.W, p->dct);
  } else {
    std::vector<uint8_t> lastcode = last.analytic ? pack_codes(fl, fu, fv, last.H, last.W) : last.code;
    if (!coarsest_pinv(lastcode, last.H, last.W, p->pinv)) {
      delete p;
      return fail(SG_ERR_ARG, "coarsest operator could not be factorised");
    }
  }
  // tail: the largest suffix of levels that fits one block's shared memory: open boxes up
  // to kOpenTailMaxSide cells a side (k_gmg_tail_open), otherwise up to kTailMaxSide
  // (k_gmg_tail, codes from global memory); e and b of every level plus the scratch of
  // the first one
  size_t cyc = precision == SG_GMG_FP64 ? sizeof(double) : sizeof(float);
  const int64_t budget = 220 * 1024;
  int nl = (int)p->levels.size();
  auto generic_elems = [&](int start) {
    int64_t acc = 0;
    for (int k = start; k < nl; ++k) acc += ((2 * (int64_t)p->levels[k].H * p->levels[k].W + 3) & ~(int64_t)3);
    return acc + (int64_t)p->levels[start].H * ((p->levels[start].W + 1) / 2);
  };
  p->tail_start = p->coarse_dct ? nl : nl - 1;  // no tail kernel above a cosine-transform solve
  bool open_suffix = !p->coarse_dct;
  for (int k = p->coarse_dct ? -1 : nl - 1; k >= 0; --k) {
    const Level& L = p->levels[k];
    const bool open = open_suffix && L.analytic;
    const int side = std::max(L.H, L.W);
    const int64_t elems = open ? (int64_t)open_tail_layout(p->levels, k).total : generic_elems(k);
    if (side > (open ? kOpenTailMaxSide : kTailMaxSide) || elems * (int64_t)cyc > budget) break;
    open_suffix = open;
    p->tail_start = k;
  }
  p->tail_open = open_suffix ? 1 : 0;
  if (p->coarse_dct) {
    const Level& C = p->levels.back();
    p->tail_smem = 0;
    // float64 arithmetic in FP64 and mixed precision (the coarsest solve stays FP64 there, as
    // the dense pseudo-inverse's does); mixed levels that need the four-product form (rows
    // not in 16-byte units) keep it in float32
    const bool fits = precision == SG_GMG_FP64 ? dct_stream_fits<double, double>(C)
                                               : (precision == SG_GMG_MIXED ? dct_stream_fits<float, double>(C)
                                                                           : dct_stream_fits<float, float>(C));
    p->coarse_dct_stream = p->coarse_dct_multi && fits ? 1 : 0;
    p->dct_fp64 = precision == SG_GMG_FP64 || (precision == SG_GMG_MIXED && (!p->coarse_dct_multi || fits)) ? 1 : 0;
    if (p->coarse_dct_stream) {
      const size_t sT = precision == SG_GMG_FP64 ? 8 : 4, sTA = p->dct_fp64 ? 8 : 4;
      const DctClusterLayout lf = dct_cluster_layout(false, C.H, C.W, sT, sTA);
      const DctClusterLayout li = dct_cluster_layout(true, C.H, C.W, sT, sTA);
      const size_t split_off = (2 * (size_t)C.W * C.W + (size_t)C.H * C.H + C.W + C.H) * sTA;
      const bool cfit = C.H % kDcNC == 0 && C.W % kDcNC == 0 && ((size_t)(C.W / kDcNC) * sTA) % 16 == 0 &&
                        split_off % 16 == 0 && p->dct.size() == 3 * (size_t)C.W * C.W + (size_t)C.H * C.H + C.W + C.H &&
                        std::max(lf.bytes, li.bytes) <= (size_t)kDsSmemBudget && lf.nch <= kDsMaxSlots &&
                        li.nch <= kDsMaxSlots;
      p->coarse_dct_cluster = cfit ? 1 : 0;
      p->dct_cluster_smem[0] = (int64_t)lf.bytes;
      p->dct_cluster_smem[1] = (int64_t)li.bytes;
    }
    p->dct_stream_smem = !p->coarse_dct_stream ? 0
                         : (int64_t)(p->dct_fp64 ? dct_stream_layout<double>(C.H, C.W).bytes
                                                 : dct_stream_layout<float>(C.H, C.W).bytes);
    p->dct_smem = p->coarse_dct_multi ? 0
                                      : (int64_t)(p->dct_fp64 ? coarse_dct_smem<double>(C.H, C.W)
                                                              : coarse_dct_smem<float>(C.H, C.W));
  } else {
    p->tail_smem = (p->tail_open ? (int64_t)open_tail_layout(p->levels, p->tail_start).total
                                 : generic_elems(p->tail_start)) *
                   (int64_t)cyc;
  }
  // workspace layout
  size_t fine = precision == SG_GMG_FP32 ? sizeof(float) : sizeof(double);
  int64_t off = 0;
  for (size_t k = 0; k + 1 < p->levels.size(); ++k) {
    const Level& L = p->levels[k];
    const Level& C = p->levels[k + 1];
    p->levels[k].fused = (L.analytic && C.analytic && L.H >= 2 && L.W >= 2 && pre_sweeps >= 1 && pre_sweeps <= 3 &&
                          post_sweeps >= 1 && post_sweeps <= 3)
                             ? 1
                             : 0;
  }
  for (auto& L : p->levels) {
    L.ld = ((int64_t)L.W + 31) / 32 * 32;
    int64_t n = L.ld * L.H;
    L.off_e = off;
    off = align256(off + n * (int64_t)cyc);
    L.off_e2 = off;
    if (L.fused) off = align256(off + n * (int64_t)cyc);
    L.off_b = off;
    off = align256(off + n * (int64_t)cyc);
    L.off_code = off;
    if (!L.analytic) off = align256(off + (int64_t)L.H * L.W);
  }
  p->ld_bfine = p->levels[0].ld;
  p->off_bfine = off;
  off = align256(off + p->ld_bfine * p->H * (int64_t)fine);
  p->fused_ir = (p->levels.size() >= 2 && p->tail_start >= 1 && p->levels[0].fused && !small_tiles(p->levels[0])) ? 1 : 0;
  if (p->fused_ir) {
    p->off_b2 = off;
    off = align256(off + p->levels[0].ld * p->H * (int64_t)cyc);
    if (precision == SG_GMG_MIXED) {
      p->off_r64 = off;
      off = align256(off + p->levels[0].ld * p->H * (int64_t)fine);
    }
  }
  p->off_pinv = off;
  off = align256(off + (int64_t)p->pinv.size() * 8);
  p->off_dct = off;
  off = align256(off + (int64_t)p->dct.size() * 8);
  if (p->coarse_dct_multi) {  // the products' two H x W intermediates
    p->off_dct_x = off;
    off = align256(off + 2 * (int64_t)p->levels.back().H * p->levels.back().W * (int64_t)cyc);
  }
  dim3 g = grid_wide(p->W, p->H);
  p->n_partial = (int64_t)g.x * g.y;
  if (p->fused_ir) {
    dim3 gf = precision == SG_GMG_FP64 ? post_final_grid<double>(p) : post_final_grid<float>(p);
    p->n_partial = std::max(p->n_partial, (int64_t)gf.x * gf.y);
  }
  p->off_partial = off;
  off = align256(off + p->n_partial * 8);
  p->off_state = off;
  off = align256(off + (int64_t)sizeof(GmgState));
  p->bytes = off;
  *out = p;
  return SG_OK;
}

void sg_gmg_plan_destroy(sg_gmg_plan* plan) {
  if (!plan) return;
  if (plan->exec) cudaGraphExecDestroy(plan->exec);
  if (plan->capture_stream) cudaStreamDestroy(plan->capture_stream);
  delete plan;
}

int64_t sg_gmg_workspace_bytes(const sg_gmg_plan* plan) { return plan ? plan->bytes : -1; }

int sg_gmg_num_levels(const sg_gmg_plan* plan) { return plan ? (int)plan->levels.size() : -1; }

int sg_gmg_bind(sg_gmg_plan* plan, void* workspace, void* stream) {
  SG_REQUIRE(plan && workspace, "null plan or workspace");
  SG_REQUIRE(((uintptr_t)workspace & 255) == 0, "workspace must be 256-byte aligned");
  plan->ws = (char*)workspace;
  if (plan->exec) {
    cudaGraphExecDestroy(plan->exec);
    plan->exec = nullptr;
  }
  cudaStream_t s = as_stream(stream);
  for (auto& L : plan->levels)
    if (!L.analytic)
      SG_CUDA_TRY(cudaMemcpyAsync(plan->ws + L.off_code, L.code.data(), L.code.size(), cudaMemcpyHostToDevice, s),
                  "sg_gmg_bind codes");
  SG_CUDA_TRY(cudaMemcpyAsync(plan->ws + plan->off_pinv, plan->pinv.data(), plan->pinv.size() * 8,
                              cudaMemcpyHostToDevice, s),
              "sg_gmg_bind pinv");
  if (plan->coarse_dct) {
    if (plan->dct_fp64) {
      SG_CUDA_TRY(cudaMemcpyAsync(plan->ws + plan->off_dct, plan->dct.data(), plan->dct.size() * 8,
                                  cudaMemcpyHostToDevice, s),
                  "sg_gmg_bind cosine tables");
    } else {
      plan->dct_f.assign(plan->dct.begin(), plan->dct.end());
      SG_CUDA_TRY(cudaMemcpyAsync(plan->ws + plan->off_dct, plan->dct_f.data(), plan->dct_f.size() * 4,
                                  cudaMemcpyHostToDevice, s),
                  "sg_gmg_bind cosine tables");
    }
    const int ds = (int)plan->dct_smem;
    if (plan->coarse_dct_multi) {
      const int rc = plan->precision == SG_GMG_FP64 ? set_dct_gemm_smem<double>() : set_dct_gemm_smem<float>();
      if (rc != SG_OK) return rc;
      if (plan->coarse_dct_stream) {
        const int rc2 = plan->precision == SG_GMG_FP64 ? set_dct_stream_smem<double, double>(plan)
                        : (plan->dct_fp64 ? set_dct_stream_smem<float, double>(plan)
                                          : set_dct_stream_smem<float, float>(plan));
        if (rc2 != SG_OK) return rc2;
      }
    }
    if (!plan->coarse_dct_multi)
      SG_CUDA_TRY(plan->precision == SG_GMG_FP64
                      ? cudaFuncSetAttribute(k_gmg_coarse_dct<double, double>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, ds)
                      : (plan->dct_fp64 ? cudaFuncSetAttribute(k_gmg_coarse_dct<float, double>,
                                                               cudaFuncAttributeMaxDynamicSharedMemorySize, ds)
                                        : cudaFuncSetAttribute(k_gmg_coarse_dct<float, float>,
                                                               cudaFuncAttributeMaxDynamicSharedMemorySize, ds)),
                  "smem attr");
  }
  SG_CUDA_TRY(cudaMemsetAsync(plan->ws + plan->off_state, 0, sizeof(GmgState), s), "sg_gmg_bind state");
  // host vectors must outlive the asynchronous copies
  SG_CUDA_TRY(cudaStreamSynchronize(s), "sg_gmg_bind sync");
  int rc = plan->precision == SG_GMG_FP64 ? set_tiled_smem_limits<double>() : set_tiled_smem_limits<float>();
  if (rc != SG_OK) return rc;
  int smem = (int)plan->tail_smem;
  if (plan->precision == SG_GMG_FP64) {
    SG_CUDA_TRY(cudaFuncSetAttribute(k_gmg_tail<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem), "smem attr");
    SG_CUDA_TRY(cudaFuncSetAttribute(k_gmg_tail_open<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem),
                "smem attr");
  } else {
    SG_CUDA_TRY(cudaFuncSetAttribute(k_gmg_tail<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem), "smem attr");
    SG_CUDA_TRY(cudaFuncSetAttribute(k_gmg_tail_open<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem),
                "smem attr");
  }
  return SG_OK;
}

#define SG_GMG_TYPED(call_fp32_f32, ...)                                                           \
  do {                                                                                             \
    bool d32 = div_dtype == SG_F32;                                                                \
    switch (plan->precision) {                                                                     \
      case SG_GMG_FP32:                                                                            \
        if (d32) return call_fp32_f32<float, float, float>(__VA_ARGS__);                           \
        return call_fp32_f32<float, double, float>(__VA_ARGS__);                                   \
      case SG_GMG_FP64:                                                                            \
        if (d32) return call_fp32_f32<double, float, double>(__VA_ARGS__);                         \
        return call_fp32_f32<double, double, double>(__VA_ARGS__);                                 \
      default:                                                                                     \
        if (d32) return call_fp32_f32<double, float, float>(__VA_ARGS__);                          \
        return call_fp32_f32<double, double, float>(__VA_ARGS__);                                  \
    }                                                                                              \
  } while (0)

static int check_solve_args(sg_gmg_plan* plan, void* p, int64_t ld_p, const void* div, int64_t ld_div, int div_dtype) {
  SG_REQUIRE(plan && plan->ws, "plan not bound to a workspace");
  SG_REQUIRE(p && div && ld_p >= plan->W && ld_div >= plan->W, "bad pressure/divergence");
  SG_REQUIRE(div_dtype == SG_F32 || div_dtype == SG_F64, "bad div dtype");
  return SG_OK;
}

int sg_gmg_solve_async(sg_gmg_plan* plan, void* p, int64_t ld_p, const void* div, int64_t ld_div, int div_dtype,
                       double alpha, double tol, int max_cycles, void* stream) {
  int rc = check_solve_args(plan, p, ld_p, div, ld_div, div_dtype);
  if (rc != SG_OK) return rc;
  SG_REQUIRE(max_cycles >= 0 && max_cycles < kHist, "max_cycles must be in 0..%d", kHist - 1);
  cudaStream_t s = as_stream(stream);
  SG_GMG_TYPED(solve_async_typed, plan, p, ld_p, div, ld_div, alpha, tol, max_cycles, s, false);
}

int sg_gmg_solve_from_zero_async(sg_gmg_plan* plan, void* p, int64_t ld_p, const void* div, int64_t ld_div,
                                 int div_dtype, double alpha, double tol, int max_cycles, void* stream) {
  int rc = check_solve_args(plan, p, ld_p, div, ld_div, div_dtype);
  if (rc != SG_OK) return rc;
  SG_REQUIRE(max_cycles >= 0 && max_cycles < kHist, "max_cycles must be in 0..%d", kHist - 1);
  cudaStream_t s = as_stream(stream);
  SG_GMG_TYPED(solve_async_typed, plan, p, ld_p, div, ld_div, alpha, tol, max_cycles, s, true);
}

int sg_gmg_stats(sg_gmg_plan* plan, int* cycles, double* relres, int* status, long long* total_cycles, void* stream) {
  SG_REQUIRE(plan && plan->ws, "plan not bound to a workspace");
  GmgState st;
  SG_CUDA_TRY(cudaMemcpyAsync(&st, state_ptr(plan), sizeof(GmgState), cudaMemcpyDeviceToHost, as_stream(stream)),
              "sg_gmg_stats copy");
  SG_CUDA_TRY(cudaStreamSynchronize(as_stream(stream)), "sg_gmg_stats sync");
  if (cycles) *cycles = st.cycles;
  if (relres) *relres = st.relres;
  if (status) *status = st.status;
  if (total_cycles) *total_cycles = st.total_cycles;
  return SG_OK;
}

int sg_gmg_relres_async(sg_gmg_plan* plan, double* dst, void* stream) {
  SG_REQUIRE(plan && plan->ws && dst, "plan not bound / null destination");
  SG_CUDA_TRY(cudaMemcpyAsync(dst, &state_ptr(plan)->relres, sizeof(double), cudaMemcpyDefault, as_stream(stream)),
              "sg_gmg_relres_async");
  return SG_OK;
}

int sg_gmg_counters(sg_gmg_plan* plan, long long* solves, long long* cycles, long long* failures, void* stream) {
  SG_REQUIRE(plan && plan->ws, "plan not bound to a workspace");
  GmgState st;
  SG_CUDA_TRY(cudaMemcpyAsync(&st, state_ptr(plan), sizeof(GmgState), cudaMemcpyDeviceToHost, as_stream(stream)),
              "sg_gmg_counters copy");
  SG_CUDA_TRY(cudaStreamSynchronize(as_stream(stream)), "sg_gmg_counters sync");
  if (solves) *solves = st.solves;
  if (cycles) *cycles = st.total_cycles;
  if (failures) *failures = st.failures;
  return SG_OK;
}

int sg_gmg_solve(sg_gmg_plan* plan, void* p, int64_t ld_p, const void* div, int64_t ld_div, int div_dtype, double alpha,
                 double tol, int max_cycles, int* cycles_out, double* relres_out, void* stream) {
  int rc = sg_gmg_solve_async(plan, p, ld_p, div, ld_div, div_dtype, alpha, tol, max_cycles, stream);
  if (rc != SG_OK) return rc;
  int cycles = 0, status = 0;
  double rel = 0.0;
  rc = sg_gmg_stats(plan, &cycles, &rel, &status, nullptr, stream);
  if (rc != SG_OK) return rc;
  if (cycles_out) *cycles_out = cycles;
  if (relres_out) *relres_out = rel;
  if (status == 3) return fail(SG_ERR_NONFINITE, "non-finite residual after %d cycles", cycles);
  if (status == 4) return fail(SG_ERR_CUDA, "a bounded device wait of the solve gave up (bulk copy never landed)");
  if (status != 1)
    return fail(SG_ERR_NOT_CONVERGED, "relative residual %.3e > tol %.3e after %d cycles", rel, tol, cycles);
  return SG_OK;
}

int sg_gmg_cycles_async(sg_gmg_plan* plan, void* p, int64_t ld_p, const void* div, int64_t ld_div, int div_dtype,
                        double alpha, int n_cycles, double* relres_dev, void* stream) {
  int rc = check_solve_args(plan, p, ld_p, div, ld_div, div_dtype);
  if (rc != SG_OK) return rc;
  SG_REQUIRE(relres_dev, "relres_dev required");
  SG_REQUIRE(n_cycles >= 0 && n_cycles < kHist, "n_cycles must be in 0..%d", kHist - 1);
  cudaStream_t s = as_stream(stream);
  SG_GMG_TYPED(cycles_typed, plan, p, ld_p, div, ld_div, alpha, n_cycles, relres_dev, s);
}

int sg_gmg_graph_nodes(const sg_gmg_plan* plan, int* prologue_nodes, int* body_nodes) {
  SG_REQUIRE(plan, "null plan");
  if (prologue_nodes) *prologue_nodes = plan->prologue_nodes;
  if (body_nodes) *body_nodes = plan->body_nodes;
  return SG_OK;
}

int sg_gmg_level_shape(const sg_gmg_plan* plan, int level, int* H, int* W) {
  SG_REQUIRE(plan && H && W, "null argument");
  SG_REQUIRE(level >= 0 && level < (int)plan->levels.size(), "level out of range");
  *H = plan->levels[level].H;
  *W = plan->levels[level].W;
  return SG_OK;
}

int sg_gmg_tail_start(const sg_gmg_plan* plan) { return plan ? plan->tail_start : -1; }

int sg_gmg_set_remove_mean(sg_gmg_plan* plan, int on) {
  SG_REQUIRE(plan, "null plan");
  SG_REQUIRE(on == 0 || on == 1, "on must be 0 or 1");
  if (plan->remove_mean != on && plan->exec) {  // the cached solve graph has the old prologue
    cudaGraphExecDestroy(plan->exec);
    plan->exec = nullptr;
  }
  plan->remove_mean = on;
  return SG_OK;
}

int sg_gmg_set_inner_cycles(sg_gmg_plan* plan, int inner) {
  SG_REQUIRE(plan, "null plan");
  SG_REQUIRE(inner >= 1 && inner <= 8, "inner cycles must be in 1..8");
  if (plan->inner != inner && plan->exec) {  // the cached solve graph has the old body
    cudaGraphExecDestroy(plan->exec);
    plan->exec = nullptr;
  }
  plan->inner = inner;
  return SG_OK;
}

int sg_gmg_smooth_async(sg_gmg_plan* plan, int level, int sweeps, void* stream) {
  SG_REQUIRE(plan && plan->ws, "plan not bound to a workspace");
  SG_REQUIRE(level >= 0 && level < (int)plan->levels.size() - 1, "level must be a smoothed (non-coarsest) level");
  SG_REQUIRE(sweeps >= 0, "sweeps must be >= 0");
  const Level& L = plan->levels[level];
  LevelMask m = level_mask(plan, level);
  cudaStream_t s = as_stream(stream);
  dim3 gh = grid2d((L.W + 1) / 2, L.H);
  if (plan->precision == SG_GMG_FP64) {
    double* e = ws_ptr<double>(plan, L.off_e);
    const double* b = ws_ptr<double>(plan, L.off_b);
    for (int sw = 0; sw < sweeps; ++sw)
      for (int color = 0; color < 2; ++color)
        SG_LAUNCH(k_gmg_rbgs<double><<<gh, block2d(), 0, s>>>(L.H, L.W, e, L.ld, b, m, plan->omega, color, 0));
  } else {
    float* e = ws_ptr<float>(plan, L.off_e);
    const float* b = ws_ptr<float>(plan, L.off_b);
    for (int sw = 0; sw < sweeps; ++sw)
      for (int color = 0; color < 2; ++color)
        SG_LAUNCH(k_gmg_rbgs<float><<<gh, block2d(), 0, s>>>(L.H, L.W, e, L.ld, b, m, (float)plan->omega, color, 0));
  }
  return check_launch("sg_gmg_smooth_async");
}

int sg_gmg_fine_fused(const sg_gmg_plan* plan) { return plan ? plan->fused_ir : 0; }

int sg_gmg_set_post_events(sg_gmg_plan* plan, void* const* events, int n_pairs) {
  SG_REQUIRE(plan, "null plan");
  SG_REQUIRE(n_pairs >= 0 && (n_pairs == 0 || events), "n_pairs must be >= 0 with events for each pair");
  for (int k = 0; k < 2 * n_pairs; ++k) SG_REQUIRE(events[k], "event %d is NULL", k);
  plan->post_ev.assign(reinterpret_cast<const cudaEvent_t*>(events),
                       reinterpret_cast<const cudaEvent_t*>(events) + 2 * (size_t)n_pairs);
  plan->post_ev_next = 0;
  return SG_OK;
}

int sg_gmg_coarse_solve_kind(const sg_gmg_plan* plan) {
  if (!plan) return -1;
  if (!plan->coarse_dct) return 0;
  return plan->coarse_dct_cluster ? 4 : (plan->coarse_dct_stream ? 3 : (plan->coarse_dct_multi ? 2 : 1));
}

int sg_gmg_fine_kernel_async(sg_gmg_plan* plan, int which, void* p, int64_t ld_p, void* stream) {
  SG_REQUIRE(plan && plan->ws, "plan not bound to a workspace");
  SG_REQUIRE(plan->fused_ir, "the fine level of this plan does not run the fused kernels");
  SG_REQUIRE(which == 0 || which == 1, "which must be 0 (pre) or 1 (post)");
  SG_REQUIRE(which == 0 || (p && ld_p >= plan->W), "post kernel needs the pressure array");
  cudaStream_t s = as_stream(stream);
  auto pre = [&](auto tag) {
    using TC = decltype(tag);
    const TC* b_alt = ws_ptr<TC>(plan, plan->off_b2);
    switch (plan->pre) {
      case 1: launch_pre_reg<TC, 1>(plan, 0, true, s, b_alt); break;
      case 2: launch_pre_reg<TC, 2>(plan, 0, true, s, b_alt); break;
      default: launch_pre_reg<TC, 3>(plan, 0, true, s, b_alt); break;
    }
  };
  auto post = [&](auto tc, auto tp) {
    using TC = decltype(tc);
    using TP = decltype(tp);
    switch (plan->post) {
      case 1: launch_post_final<TC, TP, 1>(plan, (TP*)p, ld_p, s); break;
      case 2: launch_post_final<TC, TP, 2>(plan, (TP*)p, ld_p, s); break;
      default: launch_post_final<TC, TP, 3>(plan, (TP*)p, ld_p, s); break;
    }
  };
  if (plan->precision == SG_GMG_FP64) {
    if (which == 0) pre(0.0); else post(0.0, 0.0);
  } else if (plan->precision == SG_GMG_MIXED) {
    if (which == 0) pre(0.0f); else post(0.0f, 0.0);
  } else {
    if (which == 0) pre(0.0f); else post(0.0f, 0.0f);
  }
  return check_launch("sg_gmg_fine_kernel_async");
}

}  // extern "C"

SG_BOUNDS_ACCESSOR(gmg)
