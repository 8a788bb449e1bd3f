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

#include <algorithm>
#include <cstring>
#include <vector>

#include "common.cuh"

namespace sg {

// Per-cell code of a level: bit0 fluid, bit1 left face open, bit2 right, bit3 down, bit4 up.
enum : uint8_t { C_FLUID = 1, C_L = 2, C_R = 4, C_D = 8, C_U = 16 };

struct LevelMask {
  const uint8_t* code;  // planes mode only
  int64_t ld;
  int analytic;  // 1: all cells fluid and every interior face open
  int H, W;
  __device__ __forceinline__ uint8_t get(int j, int i) const {
    if (!analytic) return code[(int64_t)j * ld + i];
    uint8_t c = C_FLUID;
    if (i > 0) c |= C_L;
    if (i < W - 1) c |= C_R;
    if (j > 0) c |= C_D;
    if (j < H - 1) c |= C_U;
    return c;
  }
  __device__ __forceinline__ bool fluid(int j, int i) const { return analytic ? true : (code[(int64_t)j * ld + i] & C_FLUID); }
};

// ---------------------------------------------------------------- kernels
// Red-black Gauss-Seidel half sweep with the exact diagonal and over-relaxation.
template <typename T>
__global__ void k_gmg_rbgs(int H, int W, T* __restrict__ e, int64_t ld, const T* __restrict__ b, LevelMask m, T omega,
                           int color) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  int i = 2 * k + ((j + color) & 1);
  if (i >= W || j >= H) return;
  uint8_t c = m.get(j, i);
  if (!(c & C_FLUID)) return;
  int64_t o = (int64_t)j * ld + i;
  T acc = b[o];
  int n = 0;
  if (c & C_L) { acc += e[o - 1]; ++n; }
  if (c & C_R) { acc += e[o + 1]; ++n; }
  if (c & C_D) { acc += e[o - ld]; ++n; }
  if (c & C_U) { acc += e[o + ld]; ++n; }
  if (n == 0) return;
  T x = e[o];
  T gs = acc / (T)n;
  e[o] = x + omega * (gs - x);
}

// r = b - A e on fluid cells (0 elsewhere), written in TO; per-block sums of r^2 (double).
template <typename T, typename TO>
__global__ void k_gmg_residual(int H, int W, const T* __restrict__ e, int64_t lde, const T* __restrict__ b,
                               int64_t ldb, LevelMask m, TO* __restrict__ r, int64_t ldr, double* __restrict__ partial) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  double sq = 0.0;
  if (i < W && j < H) {
    uint8_t c = m.get(j, i);
    T acc = (T)0;
    if (c & C_FLUID) {
      int64_t o = (int64_t)j * lde + i;
      T x = e[o];
      acc = b[(int64_t)j * ldb + i];
      if (c & C_L) acc += e[o - 1] - x;
      if (c & C_R) acc += e[o + 1] - x;
      if (c & C_D) acc += e[o - lde] - x;
      if (c & C_U) acc += e[o + lde] - x;
      sq = (double)acc * (double)acc;
    }
    if (r) r[(int64_t)j * ldr + i] = (TO)acc;
  }
  if (partial) {
    double s = block_sum(sq);
    if (threadIdx.x == 0 && threadIdx.y == 0) partial[blockIdx.y * gridDim.x + blockIdx.x] = s;
  }
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

// bc = P^T r.
template <typename T>
__global__ void k_gmg_restrict(int H, int W, const T* __restrict__ r, int64_t ldr, LevelMask fm, int Hc, int Wc,
                               T* __restrict__ bc, int64_t ldc, LevelMask cm) {
  int I = blockIdx.x * blockDim.x + threadIdx.x;
  int J = blockIdx.y * blockDim.y + threadIdx.y;
  if (I >= Wc || J >= Hc) return;
  const T w[4] = {(T)(9.0 / 16.0), (T)(3.0 / 16.0), (T)(3.0 / 16.0), (T)(1.0 / 16.0)};
  T acc = (T)0;
  if (cm.fluid(J, I)) {
    for (int j = 2 * J - 2; j <= 2 * J + 3; ++j) {
      if (j < 0 || j >= H) continue;
      for (int i = 2 * I - 2; i <= 2 * I + 3; ++i) {
        if (i < 0 || i >= W || !fm.fluid(j, i)) continue;
        int cj[4], ci[4];
        pcand(j, i, Hc, Wc, cm, cj, ci);
        T rv = r[(int64_t)j * ldr + i];
#pragma unroll
        for (int q = 0; q < 4; ++q)
          if (cj[q] == J && ci[q] == I) acc += w[q] * rv;
      }
    }
  }
  bc[(int64_t)J * ldc + I] = acc;
}

// e += P ec on fluid fine cells.
template <typename T>
__global__ void k_gmg_prolong_add(int Hc, int Wc, const T* __restrict__ ec, int64_t ldc, LevelMask cm, int H, int W,
                                  T* __restrict__ e, int64_t lde, LevelMask fm) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= W || j >= H) return;
  if (!fm.fluid(j, i)) return;
  const T w[4] = {(T)(9.0 / 16.0), (T)(3.0 / 16.0), (T)(3.0 / 16.0), (T)(1.0 / 16.0)};
  int cj[4], ci[4];
  pcand(j, i, Hc, Wc, cm, cj, ci);
  T acc = (T)0;
#pragma unroll
  for (int q = 0; q < 4; ++q) acc += w[q] * ec[(int64_t)cj[q] * ldc + ci[q]];
  e[(int64_t)j * lde + i] += acc;
}

// Exact coarsest solve e = A^+ b (one block; pinv is n x n doubles, n = H * W).
template <typename T>
__global__ void k_gmg_coarse_solve(int H, int W, const T* __restrict__ b, int64_t ldb, T* __restrict__ e, int64_t lde,
                                   const double* __restrict__ pinv) {
  extern __shared__ double sb[];
  int n = H * W;
  for (int k = threadIdx.x; k < n; k += blockDim.x) sb[k] = (double)b[(int64_t)(k / W) * ldb + (k % W)];
  __syncthreads();
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    const double* row = pinv + (int64_t)k * n;
    double acc = 0.0;
    for (int q = 0; q < n; ++q) acc += row[q] * sb[q];
    e[(int64_t)(k / W) * lde + (k % W)] = (T)acc;
  }
}

// b = alpha * div (in the fine precision) plus per-block sums of b^2.
template <typename TD, typename TB>
__global__ void k_gmg_rhs(int H, int W, const TD* __restrict__ div, int64_t ldd, double alpha, LevelMask m,
                          TB* __restrict__ b, int64_t ldb, double* __restrict__ partial) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  double sq = 0.0;
  if (i < W && j < H) {
    TB v = (TB)0;
    if (m.fluid(j, i)) {
      v = (TB)(alpha * (double)div[(int64_t)j * ldd + i]);
      sq = (double)v * (double)v;
    }
    b[(int64_t)j * ldb + i] = v;
  }
  double s = block_sum(sq);
  if (threadIdx.x == 0 && threadIdx.y == 0) partial[blockIdx.y * gridDim.x + blockIdx.x] = s;
}

// p += e (fine precision += cycle precision).
template <typename TP, typename TE>
__global__ void k_gmg_correct(int H, int W, TP* __restrict__ p, int64_t ldp, const TE* __restrict__ e, int64_t lde) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= W || j >= H) return;
  p[(int64_t)j * ldp + i] += (TP)e[(int64_t)j * lde + i];
}

// Deterministic final sum of block partials; out = sqrt(sum) (mode 0) or
// out = sqrt(sum) / nb[0] (mode 1, relative to a stored norm); NaN/Inf flags status.
__global__ void k_gmg_finalize(const double* __restrict__ partial, int n, double* __restrict__ out,
                               const double* __restrict__ nb, int mode) {
  double s = 0.0;
  for (int k = threadIdx.x; k < n; k += blockDim.x) s += partial[k];
  __shared__ double red[1024];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    double v = sqrt(red[0]);
    if (mode == 1) {
      double n = nb[0];
      if (!(n == n) || isinf(n)) v = n + v;  // a non-finite ||b|| makes the ratio non-finite
      else v = n > 0.0 ? v / n : 0.0;
    }
    out[0] = v;
  }
}

// ---------------------------------------------------------------- plan
struct Level {
  int H = 0, W = 0;
  int64_t ld = 0;        // row stride of the real arrays
  int analytic = 0;      // every cell fluid and every interior face open
  std::vector<uint8_t> code;  // H * W codes (host), empty when analytic
  int64_t off_e = 0, off_b = 0, off_r = 0, off_code = 0;
};

}  // namespace sg

struct sg_gmg_plan {
  int H, W, precision, cycle, pre, post, coarsest;
  double omega;
  std::vector<sg::Level> levels;
  std::vector<double> pinv;  // coarsest pseudo-inverse, n x n
  int64_t off_pinv, off_bfine, off_partial, off_scalars, bytes;
  int64_t ld_bfine;
  int64_t n_partial;
  char* ws;  // bound device workspace
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
  // connected components over open faces
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
  // Gauss-Jordan inversion with partial pivoting
  std::vector<double> I((size_t)n * n, 0.0);
  for (int a = 0; a < n; ++a) I[(size_t)a * n + a] = 1.0;
  for (int col = 0; col < n; ++col) {
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

static LevelMask level_mask(const sg_gmg_plan* p, int k) {
  const Level& L = p->levels[k];
  LevelMask m;
  m.code = L.analytic ? nullptr : (const uint8_t*)(p->ws + L.off_code);
  m.ld = L.W;
  m.analytic = L.analytic;
  m.H = L.H;
  m.W = L.W;
  return m;
}

template <typename T>
static T* lvl_ptr(const sg_gmg_plan* p, int64_t off) {
  return (T*)(p->ws + off);
}

// One cycle on level k: e_k updated in place for A_k e_k = b_k.
template <typename T>
static void cycle(const sg_gmg_plan* p, int k, cudaStream_t s) {
  const Level& L = p->levels[k];
  LevelMask m = level_mask(p, k);
  T* e = lvl_ptr<T>(p, L.off_e);
  T* b = lvl_ptr<T>(p, L.off_b);
  int nl = (int)p->levels.size();
  if (k == nl - 1) {
    int n = L.H * L.W;
    SG_LAUNCH(k_gmg_coarse_solve<T><<<1, 256, n * sizeof(double), s>>>(L.H, L.W, b, L.ld, e, L.ld,
                                                             (const double*)(p->ws + p->off_pinv)));
    return;
  }
  const Level& C = p->levels[k + 1];
  LevelMask cm = level_mask(p, k + 1);
  dim3 gh = grid2d((L.W + 1) / 2, L.H);
  for (int sw = 0; sw < p->pre; ++sw)
    for (int color = 0; color < 2; ++color)
      SG_LAUNCH(k_gmg_rbgs<T><<<gh, block2d(), 0, s>>>(L.H, L.W, e, L.ld, b, m, (T)p->omega, color));
  T* r = lvl_ptr<T>(p, L.off_r);
  SG_LAUNCH(k_gmg_residual<T, T><<<grid2d(L.W, L.H), block2d(), 0, s>>>(L.H, L.W, e, L.ld, b, L.ld, m, r, L.ld, nullptr));
  T* bc = lvl_ptr<T>(p, C.off_b);
  T* ec = lvl_ptr<T>(p, C.off_e);
  SG_LAUNCH(k_gmg_restrict<T><<<grid2d(C.W, C.H), block2d(), 0, s>>>(L.H, L.W, r, L.ld, m, C.H, C.W, bc, C.ld, cm));
  cudaMemsetAsync(ec, 0, sizeof(T) * C.ld * C.H, s);
  int reps = (p->cycle == 1 && k + 1 < nl - 1) ? 2 : 1;
  for (int q = 0; q < reps; ++q) cycle<T>(p, k + 1, s);
  SG_LAUNCH(k_gmg_prolong_add<T><<<grid2d(L.W, L.H), block2d(), 0, s>>>(C.H, C.W, ec, C.ld, cm, L.H, L.W, e, L.ld, m));
  for (int sw = 0; sw < p->post; ++sw)
    for (int color = 0; color < 2; ++color)
      SG_LAUNCH(k_gmg_rbgs<T><<<gh, block2d(), 0, s>>>(L.H, L.W, e, L.ld, b, m, (T)p->omega, color));
}

// Fine-level residual r = bfine - A p -> cycle rhs b_0 (+ norm into scalars[slot]).
template <typename TP, typename TC>
static void fine_residual(const sg_gmg_plan* p, const TP* pp, int64_t ldp, double* out, cudaStream_t s) {
  const Level& L = p->levels[0];
  LevelMask m = level_mask(p, 0);
  double* part = (double*)(p->ws + p->off_partial);
  double* scal = (double*)(p->ws + p->off_scalars);
  dim3 g = grid2d(L.W, L.H);
  SG_LAUNCH(k_gmg_residual<TP, TC><<<g, block2d(), 0, s>>>(L.H, L.W, pp, ldp, (const TP*)(p->ws + p->off_bfine), p->ld_bfine, m,
                                                 lvl_ptr<TC>(p, L.off_b), L.ld, part));
  SG_LAUNCH(k_gmg_finalize<<<1, 1024, 0, s>>>(part, (int)(g.x * g.y), out, scal, 1));
}

template <typename TP, typename TD, typename TC>
static int solve_impl(sg_gmg_plan* p, TP* pp, int64_t ldp, const TD* div, int64_t ldd, double alpha, double tol,
                      int max_cycles, int check_every, int* cycles_out, double* relres_out, double* relres_dev,
                      int fixed_cycles, cudaStream_t s) {
  const Level& L = p->levels[0];
  LevelMask m = level_mask(p, 0);
  double* part = (double*)(p->ws + p->off_partial);
  double* scal = (double*)(p->ws + p->off_scalars);  // [0] = ||b||, [1] = relres
  dim3 g = grid2d(L.W, L.H);
  SG_LAUNCH(k_gmg_rhs<TD, TP><<<g, block2d(), 0, s>>>(L.H, L.W, div, ldd, alpha, m, (TP*)(p->ws + p->off_bfine), p->ld_bfine, part));
  SG_LAUNCH(k_gmg_finalize<<<1, 1024, 0, s>>>(part, (int)(g.x * g.y), scal, nullptr, 0));
  double* res_slot = relres_dev ? relres_dev : scal + 1;
  fine_residual<TP, TC>(p, pp, ldp, res_slot, s);
  TC* e0 = lvl_ptr<TC>(p, L.off_e);
  int cycles = 0;
  double rel = 0.0;
  int n = fixed_cycles >= 0 ? fixed_cycles : max_cycles;
  if (fixed_cycles < 0) {
    if (cudaMemcpyAsync(&rel, res_slot, sizeof(double), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
      return check_launch("sg_gmg_solve");
    if (!(rel == rel) || std::isinf(rel)) return fail(SG_ERR_NONFINITE, "non-finite initial residual");
    if (rel <= tol) n = 0;
  }
  for (int c = 0; c < n; ++c) {
    cudaMemsetAsync(e0, 0, sizeof(TC) * L.ld * L.H, s);
    cycle<TC>(p, 0, s);
    SG_LAUNCH(k_gmg_correct<TP, TC><<<g, block2d(), 0, s>>>(L.H, L.W, pp, ldp, e0, L.ld));
    ++cycles;
    double* slot = relres_dev ? relres_dev + cycles : scal + 1;
    fine_residual<TP, TC>(p, pp, ldp, slot, s);
    if (fixed_cycles < 0 && (cycles % check_every == 0 || cycles == n)) {
      if (cudaMemcpyAsync(&rel, slot, sizeof(double), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
          cudaStreamSynchronize(s) != cudaSuccess)
        return check_launch("sg_gmg_solve");
      if (!(rel == rel) || std::isinf(rel)) return fail(SG_ERR_NONFINITE, "non-finite residual after %d cycles", cycles);
      if (rel <= tol) break;
    }
  }
  int rc = check_launch("sg_gmg_solve");
  if (rc != SG_OK) return rc;
  if (cycles_out) *cycles_out = cycles;
  if (relres_out) *relres_out = rel;
  if (fixed_cycles < 0 && rel > tol)
    return fail(SG_ERR_NOT_CONVERGED, "relative residual %.3e > tol %.3e after %d cycles", rel, tol, cycles);
  return SG_OK;
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
  SG_REQUIRE(coarsest >= 1 && coarsest <= 16, "coarsest must be in 1..16");
  SG_REQUIRE(omega > 0.0 && omega < 2.0, "omega must be in (0, 2)");
  SG_REQUIRE(pre_sweeps >= 0 && post_sweeps >= 0 && pre_sweeps + post_sweeps >= 1, "need at least one smoothing sweep");
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
  p->ws = nullptr;
  int h = (int)H, w = (int)W;
  while (true) {
    Level L;
    L.H = h;
    L.W = w;
    L.analytic = level_is_open(fl, fu, fv, h, w) ? 1 : 0;
    if (!L.analytic) L.code = pack_codes(fl, fu, fv, h, w);
    p->levels.push_back(L);
    if (std::max(h, w) <= coarsest) break;
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
  Level& last = p->levels.back();
  std::vector<uint8_t> lastcode = last.analytic ? pack_codes(fl, fu, fv, last.H, last.W) : last.code;
  if (!coarsest_pinv(lastcode, last.H, last.W, p->pinv)) {
    delete p;
    return fail(SG_ERR_ARG, "coarsest operator could not be factorised");
  }
  // workspace layout
  size_t cyc = precision == SG_GMG_FP64 ? sizeof(double) : sizeof(float);
  size_t fine = precision == SG_GMG_FP32 ? sizeof(float) : sizeof(double);
  int64_t off = 0;
  for (auto& L : p->levels) {
    L.ld = ((int64_t)L.W + 31) / 32 * 32;
    int64_t n = L.ld * L.H;
    L.off_e = off;
    off = align256(off + n * (int64_t)cyc);
    L.off_b = off;
    off = align256(off + n * (int64_t)cyc);
    L.off_r = off;
    off = align256(off + n * (int64_t)cyc);
    L.off_code = off;
    if (!L.analytic) off = align256(off + (int64_t)L.H * L.W);
  }
  p->ld_bfine = p->levels[0].ld;
  p->off_bfine = off;
  off = align256(off + p->ld_bfine * p->H * (int64_t)fine);
  p->off_pinv = off;
  off = align256(off + (int64_t)p->pinv.size() * 8);
  dim3 g = grid2d(p->W, p->H);
  p->n_partial = (int64_t)g.x * g.y;
  p->off_partial = off;
  off = align256(off + p->n_partial * 8);
  p->off_scalars = off;
  off = align256(off + 8 * 8);
  p->bytes = off;
  *out = p;
  return SG_OK;
}

void sg_gmg_plan_destroy(sg_gmg_plan* plan) { delete plan; }

int64_t sg_gmg_workspace_bytes(const sg_gmg_plan* plan) { return plan ? plan->bytes : -1; }

int sg_gmg_num_levels(const sg_gmg_plan* plan) { return plan ? (int)plan->levels.size() : -1; }

int sg_gmg_bind(sg_gmg_plan* plan, void* workspace, void* stream) {
  SG_REQUIRE(plan && workspace, "null plan or workspace");
  SG_REQUIRE(((uintptr_t)workspace & 255) == 0, "workspace must be 256-byte aligned");
  plan->ws = (char*)workspace;
  cudaStream_t s = as_stream(stream);
  for (auto& L : plan->levels)
    if (!L.analytic) {
      cudaError_t e = cudaMemcpyAsync(plan->ws + L.off_code, L.code.data(), L.code.size(), cudaMemcpyHostToDevice, s);
      if (e != cudaSuccess) return fail(SG_ERR_CUDA, "sg_gmg_bind: %s", cudaGetErrorString(e));
    }
  cudaError_t e = cudaMemcpyAsync(plan->ws + plan->off_pinv, plan->pinv.data(), plan->pinv.size() * 8,
                                  cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) return fail(SG_ERR_CUDA, "sg_gmg_bind: %s", cudaGetErrorString(e));
  // host vectors must outlive the asynchronous copies
  e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return fail(SG_ERR_CUDA, "sg_gmg_bind: %s", cudaGetErrorString(e));
  return SG_OK;
}

static int gmg_dispatch(sg_gmg_plan* plan, void* p, int64_t ld_p, const void* div, int64_t ld_div, int div_dtype,
                        double alpha, double tol, int max_cycles, int check_every, int* cycles_out, double* relres_out,
                        double* relres_dev, int fixed, void* stream) {
  SG_REQUIRE(plan && plan->ws, "plan not bound to a workspace");
  SG_REQUIRE(p && div && ld_p >= plan->W && ld_div >= plan->W, "bad pressure/divergence");
  SG_REQUIRE(max_cycles >= 0 && check_every >= 1, "bad cycle limits");
  SG_REQUIRE(div_dtype == SG_F32 || div_dtype == SG_F64, "bad div dtype");
  cudaStream_t s = as_stream(stream);
  bool d32 = div_dtype == SG_F32;
#define SG_GMG_CALL(TP, TD, TC)                                                                                  \
  return solve_impl<TP, TD, TC>(plan, (TP*)p, ld_p, (const TD*)div, ld_div, alpha, tol, max_cycles, check_every, \
                                cycles_out, relres_out, relres_dev, fixed, s)
  switch (plan->precision) {
    case SG_GMG_FP32:
      if (d32) SG_GMG_CALL(float, float, float);
      SG_GMG_CALL(float, double, float);
    case SG_GMG_FP64:
      if (d32) SG_GMG_CALL(double, float, double);
      SG_GMG_CALL(double, double, double);
    default:
      if (d32) SG_GMG_CALL(double, float, float);
      SG_GMG_CALL(double, double, float);
  }
#undef SG_GMG_CALL
}

int sg_gmg_solve(sg_gmg_plan* plan, void* p, int64_t ld_p, const void* div, int64_t ld_div, int div_dtype, double alpha,
                 double tol, int max_cycles, int check_every, int* cycles_out, double* relres_out, void* stream) {
  return gmg_dispatch(plan, p, ld_p, div, ld_div, div_dtype, alpha, tol, max_cycles, check_every, cycles_out,
                      relres_out, nullptr, -1, stream);
}

int sg_gmg_cycles_async(sg_gmg_plan* plan, void* p, int64_t ld_p, const void* div, int64_t ld_div, int div_dtype,
                        double alpha, int n_cycles, double* relres_dev, void* stream) {
  SG_REQUIRE(relres_dev, "relres_dev required");
  SG_REQUIRE(n_cycles >= 0, "n_cycles must be >= 0");
  return gmg_dispatch(plan, p, ld_p, div, ld_div, div_dtype, alpha, 0.0, n_cycles, 1, nullptr, nullptr, relres_dev,
                      n_cycles, stream);
}

int sg_gmg_level_shape(const sg_gmg_plan* plan, int level, int* H, int* W) {
  SG_REQUIRE(plan && H && W, "null argument");
  SG_REQUIRE(level >= 0 && level < (int)plan->levels.size(), "level out of range");
  *H = plan->levels[level].H;
  *W = plan->levels[level].W;
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
    double* e = lvl_ptr<double>(plan, L.off_e);
    const double* b = lvl_ptr<double>(plan, L.off_b);
    for (int sw = 0; sw < sweeps; ++sw)
      for (int color = 0; color < 2; ++color)
        SG_LAUNCH(k_gmg_rbgs<double><<<gh, block2d(), 0, s>>>(L.H, L.W, e, L.ld, b, m, plan->omega, color));
  } else {
    float* e = lvl_ptr<float>(plan, L.off_e);
    const float* b = lvl_ptr<float>(plan, L.off_b);
    for (int sw = 0; sw < sweeps; ++sw)
      for (int color = 0; color < 2; ++color)
        SG_LAUNCH(k_gmg_rbgs<float><<<gh, block2d(), 0, s>>>(L.H, L.W, e, L.ld, b, m, (float)plan->omega, color));
  }
  return check_launch("sg_gmg_smooth_async");
}

}  // extern "C"
