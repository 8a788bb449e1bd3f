// Per-operator kernels of the smoke step and their C-ABI entry points.
//
// Each kernel restates one Numba kernel of the reference (src/cfd/backends/numba/...)
// with the same arithmetic types, so float32 and float64 results match the reference
// bit for bit (this unit is compiled with -fmad=false: no contraction into FMA).
// Launch shape: 32x8 threads, one thread per cell/face, x along the contiguous row.

#include <atomic>
#include <cstring>
#include <mutex>

#include "cell_ops.cuh"

namespace sg {

static thread_local std::string g_last_error;

void set_error(const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
}

int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

int check_launch(const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(SG_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
  return SG_OK;
}

const char* last_error_cstr() { return g_last_error.c_str(); }

static std::atomic<unsigned long long> g_launches{0};
void note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
unsigned long long launch_count() { return g_launches.load(std::memory_order_relaxed); }

// ------------------------------------------------------------------ advection
// advection.py:112-128 (+ dissipation, simulation.py:232)
template <typename T, int MM>
__global__ void k_advect_scalar(int H, int W, const T* __restrict__ src, int64_t lds, T* __restrict__ dst, int64_t ldd,
                                const T* __restrict__ u, int64_t ur, int64_t uc, int64_t ldu,
                                const T* __restrict__ v, int64_t vr, int64_t vc, int64_t ldv, MasksT<MM> m,
                                double dt, double inv, T diss) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= W) return;
#pragma unroll
  for (int q = 0; q < kRows; ++q) {
    const int j = row_of(q);
    if (j < H)
      dst[(int64_t)j * ldd + i] =
          advect_scalar_cell(j, i, H, W, src, lds, u, ur, uc, ldu, v, vr, vc, ldv, m, dt, inv, diss);
  }
}

template <typename T>
__global__ void k_advect_u(int ur, int uc, const T* __restrict__ us, int64_t ldus, T* __restrict__ ud, int64_t ldud,
                           const T* __restrict__ v, int64_t vr, int64_t vc, int64_t ldv, Masks m, double dt, double inv) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= uc || j >= ur) return;
  ud[(int64_t)j * ldud + i] = m.u(j, i) ? advect_u_face(j, i, us, ldus, ur, uc, v, vr, vc, ldv, dt, inv) : (T)0;
}

template <typename T>
__global__ void k_advect_v(int vr, int vc, const T* __restrict__ vs, int64_t ldvs, T* __restrict__ vd, int64_t ldvd,
                           const T* __restrict__ u, int64_t ur, int64_t uc, int64_t ldu, Masks m, double dt, double inv) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= vc || j >= vr) return;
  vd[(int64_t)j * ldvd + i] = m.v(j, i) ? advect_v_face(j, i, vs, ldvs, vr, vc, u, ur, uc, ldu, dt, inv) : (T)0;
}

// Both faces of the MAC grid in one launch (grid covers (W+1) x (H+1)).
template <typename T, int MM>
__global__ void k_advect_uv(int H, int W, const T* __restrict__ us, int64_t ldus, T* __restrict__ ud, int64_t ldud,
                            const T* __restrict__ vs, int64_t ldvs, T* __restrict__ vd, int64_t ldvd, MasksT<MM> m,
                            double dt, double inv) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
#pragma unroll
  for (int q = 0; q < kRows; ++q) {
  const int j = row_of(q);
  if (j < H && i <= W)
    ud[(int64_t)j * ldud + i] =
        m.u(j, i) ? advect_u_face(j, i, us, ldus, (int64_t)H, (int64_t)W + 1, vs, (int64_t)H + 1, (int64_t)W, ldvs, dt, inv)
                  : (T)0;
  if (j <= H && i < W)
    vd[(int64_t)j * ldvd + i] =
        m.v(j, i) ? advect_v_face(j, i, vs, ldvs, (int64_t)H + 1, (int64_t)W, us, (int64_t)H, (int64_t)W + 1, ldus, dt, inv)
                  : (T)0;
  }
}

// ------------------------------------------------------------------ forces
// forces.py:19-105. v is (H+1) x W.
template <typename T>
__global__ void k_apply_forces(int H, int W, T* __restrict__ v, int64_t ldv, const T* __restrict__ d, int64_t ldd,
                               const T* __restrict__ t, int64_t ldt, double dt, double g, double bc, double dc,
                               double amb, int f32tmp) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= W) return;
  // kRows consecutive faces per thread (the block's kBY * kRows rows as grid2d_rows lays them
  // out), so each thread's density rows overlap and its loads run down one column
  const int j0 = (blockIdx.y * blockDim.y + threadIdx.y) * kRows;
#pragma unroll
  for (int q = 0; q < kRows; ++q) {
    const int j = j0 + q;
    if (j <= H) forces_face(j, i, H, W, v, ldv, d, ldd, t, ldt, dt, g, bc, dc, amb, f32tmp);
  }
}

// forces.py:108-123
template <typename T>
__global__ void k_cool(int H, int W, T* __restrict__ t, int64_t ld, double amb, double decay) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= W || j >= H) return;
  int64_t k = (int64_t)j * ld + i;
  t[k] = (T)(amb + ((double)t[k] - amb) * decay);
}

// ------------------------------------------------------------------ divergence
// divergence.py:4-25
template <typename T, int MM>
__global__ void k_divergence(int H, int W, const T* __restrict__ u, int64_t ldu, const T* __restrict__ v, int64_t ldv,
                             T* __restrict__ div, int64_t ldd, MasksT<MM> m, double inv) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= W) return;
#pragma unroll
  for (int q = 0; q < kRows; ++q) {
    const int j = row_of(q);
    if (j < H) div[(int64_t)j * ldd + i] = divergence_cell(j, i, u, ldu, v, ldv, m, inv);
  }
}

// ------------------------------------------------------------------ residual
// residual.py:6-42 (+ optional sum of squares)
template <typename T, int MM>
__global__ void k_residual(int H, int W, const T* __restrict__ p, int64_t ldp, const T* __restrict__ div, int64_t ldd,
                           MasksT<MM> m, double alpha, double beta, T* __restrict__ out, int64_t ldo, double* sumsq) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double sq = 0.0;
#pragma unroll
  for (int q = 0; q < kRows; ++q) {
    const int j = row_of(q);
    if (i < W && j < H) {
      T res = residual_cell(j, i, H, W, p, ldp, div, ldd, m, alpha, beta);
      sq += (double)res * (double)res;
      if (out) out[(int64_t)j * ldo + i] = res;
    }
  }
  if (sumsq) {
    double s = block_sum(sq);
    if (threadIdx.x == 0 && threadIdx.y == 0) atomicAdd(sumsq, s);
  }
}

// ------------------------------------------------------------------ projection
// pressure_gradient.py:4-37 then, if solid_mode != SG_MASK_NONE, boundaries.py:7-39.
template <typename T, int MM, int SM>
__global__ void k_project(int H, int W, T* __restrict__ u, int64_t ldu, T* __restrict__ v, int64_t ldv,
                          const T* __restrict__ p, int64_t ldp, MasksT<MM> m, int do_grad, int solid_mode,
                          const uint8_t* __restrict__ solid, int64_t lds, double scale) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
#pragma unroll
  for (int q = 0; q < kRows; ++q)
    project_faces<T, MasksT<MM>, SM>(row_of(q), i, H, W, u, ldu, v, ldv, p, ldp, m, do_grad, solid_mode, solid, lds,
                                     scale);
}

// The substep's tail in one pass (simulation.py:244-265): the projection of (ui, vi) into
// (uo, vo) (out of place), the divergence of the projected field and the reference residual
// of p. A warp owns 32 consecutive columns and walks kTailRows rows down them: the pressure
// of the next row and the v face above the current row are computed one row ahead and
// carried in registers, the horizontal neighbours (p at i -+ 1, the u face at i + 1) come
// from the adjacent lane, so each face is projected once (plus one u face per warp edge and
// row). Every value is formed by the same expressions as the separate passes, so the
// results are identical to them.
constexpr int kTailRows = 4;

template <typename T, int MM, int SM>
__global__ void __launch_bounds__(kBX * kBY) k_project_metrics(
    int H, int W, const T* __restrict__ ui, int64_t ldui, const T* __restrict__ vi, int64_t ldvi, T* __restrict__ uo,
    int64_t lduo, T* __restrict__ vo, int64_t ldvo, const T* __restrict__ p, int64_t ldp, MasksT<MM> m, int solid_mode,
    const uint8_t* __restrict__ solid, int64_t lds, double scale, T* __restrict__ div, int64_t ldd, double inv,
    double alpha, double beta, T* __restrict__ res, int64_t ldr) {
  using MK = MasksT<MM>;
  const int lane = threadIdx.x;  // blockDim.x == 32: a warp is one row segment
  const int i = blockIdx.x * kBX + lane;
  const int j0 = (blockIdx.y * kBY + threadIdx.y) * kTailRows;
  if (j0 >= H) return;  // uniform over the warp
  const bool cell = i < W, ucol = i <= W;
  const T* pc_col = p + i;
  T p_dn = (cell && j0 > 0) ? pc_col[(int64_t)(j0 - 1) * ldp] : (T)0;
  T p_c = cell ? pc_col[(int64_t)j0 * ldp] : (T)0;
  T v_lo = (T)0;  // projected v face (j, i) of the current row
  if (cell) {
    v_lo = projected_v_pv<T, MK, SM>(j0, i, H, W, vi[(int64_t)j0 * ldvi + i], p_c, p_dn, m, solid_mode, solid, lds,
                                     scale);
    if (j0 == 0) vo[i] = v_lo;
  }
  const int jend = min(j0 + kTailRows, H);
#pragma unroll 2
  for (int j = j0; j < jend; ++j) {
    const T p_up = (cell && j + 1 < H) ? pc_col[(int64_t)(j + 1) * ldp] : (T)0;
    const T uin = ucol ? ui[(int64_t)j * ldui + i] : (T)0;
    const T vin = cell ? vi[(int64_t)(j + 1) * ldvi + i] : (T)0;
    T p_l = __shfl_up_sync(0xffffffffu, p_c, 1);
    T p_r = __shfl_down_sync(0xffffffffu, p_c, 1);
    if (lane == 0) p_l = (i > 0 && i - 1 < W) ? pc_col[(int64_t)j * ldp - 1] : (T)0;
    if (lane == kBX - 1) p_r = (i + 1 < W) ? pc_col[(int64_t)j * ldp + 1] : (T)0;
    T ul = (T)0;
    if (ucol) {
      ul = projected_u_pv<T, MK, SM>(j, i, H, W, uin, p_c, p_l, m, solid_mode, solid, lds, scale);
      uo[(int64_t)j * lduo + i] = ul;
    }
    T ur = __shfl_down_sync(0xffffffffu, ul, 1);
    if (lane == kBX - 1 && i + 1 <= W)
      ur = projected_u_pv<T, MK, SM>(j, i + 1, H, W, ui[(int64_t)j * ldui + i + 1], p_r, p_c, m, solid_mode, solid,
                                     lds, scale);
    if (cell) {
      const T v_hi = projected_v_pv<T, MK, SM>(j + 1, i, H, W, vin, p_up, p_c, m, solid_mode, solid, lds, scale);
      vo[(int64_t)(j + 1) * ldvo + i] = v_hi;
      const T dval = divergence_from_faces<T, MK>(j, i, ul, ur, v_lo, v_hi, m, inv);
      div[(int64_t)j * ldd + i] = dval;
      res[(int64_t)j * ldr + i] = residual_from_values<T, MK>(j, i, H, W, p_c, p_l, p_r, p_dn, p_up, dval, m, alpha,
                                                               beta);
      v_lo = v_hi;
    }
    p_dn = p_c;
    p_c = p_up;
  }
}

// ------------------------------------------------------------------ sources
// emitters.py:6-66 over the emitter's bounding box (x0, y0 offset).
template <typename T>
__global__ void k_emit(int bw, int bh, int x0, int y0, T* __restrict__ f, int64_t ld, double value, double dt, double px,
                       double py, double radius, int approach) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= bw || j >= bh) return;
  int x = x0 + i, y = y0 + j;
  double dx = (double)x - px, dy = (double)y - py;
  double dist = sqrt(dx * dx + dy * dy);
  if (!(dist < radius)) return;
  double fo;
  if (approach == 0) {
    fo = 1.0;
  } else if (approach == 1) {
    fo = 1.0 - dist / radius;
  } else if (approach == 2) {
    fo = 1.0 - (dist / radius) * (dist / radius);
  } else {
    double s = radius / 3.0;
    fo = exp(-0.5 * (dist / s) * (dist / s));
  }
  int64_t k = (int64_t)y * ld + x;
  f[k] = (T)((double)f[k] + value * fo * dt);
}

// Source table passed by value in the launch parameters.
constexpr int kMaxPlumes = 32;
struct PlumeTable {
  int n;
  int x0, y0;  // origin of the launch box (cells / faces)
  double row[kMaxPlumes * 6];
};

// Overwriting disc sources over the union bounding box; the last source containing a
// point wins.
template <typename T>
__global__ void k_plume(int H, int W, T* __restrict__ d, int64_t ldd, T* __restrict__ u, int64_t ldu, T* __restrict__ v,
                        int64_t ldv, const __grid_constant__ PlumeTable tab, uint64_t seed, int64_t step) {
  int i = tab.x0 + blockIdx.x * blockDim.x + threadIdx.x;
  int j = tab.y0 + blockIdx.y * blockDim.y + threadIdx.y;
  if (i > W || j > H) return;
  plume_point(j, i, H, W, d, ldd, u, ldu, v, ldv, tab.row, tab.n, seed, step);
}

// ------------------------------------------------------------------ masks
// simulation.py:103-108 from a solid plane.
__global__ void k_build_masks(int H, int W, const uint8_t* __restrict__ s, int64_t lds, uint8_t* fmu, int64_t ldu,
                              uint8_t* fmv, int64_t ldv, uint8_t* fl, int64_t ldf) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  auto S = [&](int jj, int ii) { return s[(int64_t)jj * lds + ii] != 0; };
  auto U = [&](int jj, int ii) { return ii >= 1 && ii <= W - 1 && !(S(jj, ii - 1) || S(jj, ii)); };
  auto V = [&](int jj, int ii) { return jj >= 1 && jj <= H - 1 && !(S(jj - 1, ii) || S(jj, ii)); };
  if (fmu && j < H && i <= W) fmu[(int64_t)j * ldu + i] = U(j, i) ? 1 : 0;
  if (fmv && j <= H && i < W) fmv[(int64_t)j * ldv + i] = V(j, i) ? 1 : 0;
  if (fl && j < H && i < W) fl[(int64_t)j * ldf + i] = (U(j, i) || U(j, i + 1) || V(j, i) || V(j + 1, i)) ? 1 : 0;
}

// ------------------------------------------------------------------ reference solvers
// jacobi.py:8-24
template <typename T>
__global__ void k_jacobi(int H, int W, const T* __restrict__ p, int64_t ldp, T* __restrict__ o, int64_t ldo,
                         const T* __restrict__ div, int64_t ldd, Masks m, double alpha, double rb) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= W || j >= H) return;
  T c = p[(int64_t)j * ldp + i];
  if (!m.fluid(j, i)) {
    o[(int64_t)j * ldo + i] = c;
    return;
  }
  T s = nbsum_ref(p, ldp, H, W, j, i, m, c);
  o[(int64_t)j * ldo + i] = (T)(((double)s + alpha * (double)div[(int64_t)j * ldd + i]) * rb);
}

// jacobi.py:8-24, several sweeps per launch on grids that sit in L2 (where one launch per
// sweep is launch-bound). A block stages a 16 x 32 tile plus a halo of kJG cells in shared
// memory, sweeps there with the valid region shrinking by one cell per sweep along region
// edges that are not the grid's edges, and writes its own cells: after `sweeps` <= kJG sweeps
// they hold exactly the grid-wide iterates (each update is k_jacobi's expression, in the
// same order, on the same values). Reads src, writes dst (different buffers).
constexpr int kJTR = 16, kJTC = 32, kJG = 8, kJT = 256;

template <typename T, int MM>
__global__ void __launch_bounds__(kJT) k_jacobi_tiles(int H, int W, const T* __restrict__ src, int64_t lds,
                                                      T* __restrict__ dst, int64_t ldd, const T* __restrict__ div,
                                                      int64_t lddv, MasksT<MM> m, double alpha, double rb,
                                                      int sweeps) {
  constexpr int RR = kJTR + 2 * kJG, CC = kJTC + 2 * kJG;
  __shared__ T sa[RR * CC], sb[RR * CC], sdv[RR * CC];
  const int j0 = blockIdx.y * kJTR, i0 = blockIdx.x * kJTC;
  const int R0 = max(j0 - kJG, 0), R1 = min(j0 + kJTR + kJG, H);
  const int C0 = max(i0 - kJG, 0), C1 = min(i0 + kJTC + kJG, W);
  const int nc = C1 - C0;
  for (int e = threadIdx.x; e < (R1 - R0) * nc; e += kJT) {
    const int rr = e / nc, cc = e - rr * nc;
    if (!SG_IN_BOUNDS(rr < RR && cc < CC && R0 + rr < H && C0 + cc < W)) continue;
    sa[rr * CC + cc] = src[(int64_t)(R0 + rr) * lds + C0 + cc];
    sdv[rr * CC + cc] = div[(int64_t)(R0 + rr) * lddv + C0 + cc];
  }
  __syncthreads();
  T* a = sa;
  T* b = sb;
  for (int sw = 0; sw < sweeps; ++sw) {
    const int rlo = R0 + (R0 > 0 ? sw + 1 : 0), rhi = R1 - (R1 < H ? sw + 1 : 0);
    const int clo = C0 + (C0 > 0 ? sw + 1 : 0), chi = C1 - (C1 < W ? sw + 1 : 0);
    const int w = chi - clo;
    for (int e = threadIdx.x; e < (rhi - rlo) * w; e += kJT) {
      const int j = rlo + e / w, i = clo + e % w;
      const int rr = j - R0, cc = i - C0;
      if (!SG_IN_BOUNDS(rr >= 0 && rr < RR && cc >= 0 && cc < CC && (i == 0 || i - 1 >= C0) &&
                        (i == W - 1 || i + 1 < C1) && (j == 0 || j - 1 >= R0) && (j == H - 1 || j + 1 < R1)))
        continue;
      const T c = a[rr * CC + cc];
      T out = c;
      if (m.fluid(j, i)) {
        // nbsum_ref's neighbours (clamped indices) and order, on the staged tile
        const T l = m.u(j, i) ? a[rr * CC + (max(i - 1, 0) - C0)] : c;
        const T r = m.u(j, i + 1) ? a[rr * CC + (min(i + 1, W - 1) - C0)] : c;
        const T d = m.v(j, i) ? a[(max(j - 1, 0) - R0) * CC + cc] : c;
        const T u = m.v(j + 1, i) ? a[(min(j + 1, H - 1) - R0) * CC + cc] : c;
        T sum = l + r;
        sum = sum + d;
        sum = sum + u;
        out = (T)(((double)sum + alpha * (double)sdv[rr * CC + cc]) * rb);
      }
      b[rr * CC + cc] = out;
    }
    __syncthreads();
    T* t = a;
    a = b;
    b = t;
  }
  const int jh = min(j0 + kJTR, H), ih = min(i0 + kJTC, W);
  const int ow = ih - i0;
  for (int e = threadIdx.x; e < (jh - j0) * ow; e += kJT) {
    const int j = j0 + e / ow, i = i0 + e % ow;
    if (!SG_IN_BOUNDS(j - R0 < RR && i - C0 < CC && j < H && i < W)) continue;
    dst[(int64_t)j * ldd + i] = a[(j - R0) * CC + (i - C0)];
  }
}

// red_black_sor_gauss_seidel.py:8-27, one colour: cells with (i + j) % 2 == color.
template <typename T>
__global__ void k_rbsor_half(int H, int W, T* __restrict__ p, int64_t ldp, const T* __restrict__ div, int64_t ldd,
                             Masks m, double alpha, double rb, double omega, int color) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  int i = 2 * k + ((j + color) & 1);
  if (i >= W || j >= H) return;
  if (!m.fluid(j, i)) return;
  T c = p[(int64_t)j * ldp + i];
  T s = nbsum_ref(p, ldp, H, W, j, i, m, c);
  double np_ = ((double)s + alpha * (double)div[(int64_t)j * ldd + i]) * rb;
  p[(int64_t)j * ldp + i] = (T)((1.0 - omega) * (double)c + omega * np_);
}

// gauss_seidel.py:8-26 in lexicographic order, as anti-diagonal wavefronts of one block:
// cell (j, i) reads its left/down neighbours from wavefront i+j-1 (already updated)
// and its right/up neighbours from wavefront i+j+1 (not yet updated).
template <typename T>
__global__ void k_gauss_seidel(int H, int W, T* __restrict__ p, int64_t ldp, const T* __restrict__ div, int64_t ldd,
                               Masks m, double alpha, double rb, int iterations) {
  for (int it = 0; it < iterations; ++it) {
    for (int dgl = 0; dgl <= H + W - 2; ++dgl) {
      int jlo = dgl - (W - 1) > 0 ? dgl - (W - 1) : 0;
      int jhi = dgl < H - 1 ? dgl : H - 1;
      for (int j = jlo + (int)threadIdx.x; j <= jhi; j += blockDim.x) {
        int i = dgl - j;
        if (!m.fluid(j, i)) continue;
        T c = p[(int64_t)j * ldp + i];
        T s = nbsum_ref(p, ldp, H, W, j, i, m, c);
        p[(int64_t)j * ldp + i] = (T)(((double)s + alpha * (double)div[(int64_t)j * ldd + i]) * rb);
      }
      __syncthreads();
    }
  }
}

// multigrid/transfer.py:5-36 (+ the rhs division of multigrid/solver.py:124-125)
template <typename T>
__global__ void k_restrict_avg(int H, int W, const T* __restrict__ f, int64_t ldf, Masks m, T* __restrict__ c,
                               int64_t ldc, int Hc, int Wc, T divisor) {
  int I = blockIdx.x * blockDim.x + threadIdx.x;
  int J = blockIdx.y * blockDim.y + threadIdx.y;
  if (I >= Wc || J >= Hc) return;
  double total = 0.0;
  int count = 0;
#pragma unroll
  for (int dj = 0; dj < 2; ++dj)
#pragma unroll
    for (int di = 0; di < 2; ++di) {
      int jj = 2 * J + dj, ii = 2 * I + di;
      if (m.fluid(jj, ii)) {
        total += (double)f[(int64_t)jj * ldf + ii];
        ++count;
      }
    }
  T val = count > 0 ? (T)(total / (double)count) : (T)0;
  c[(int64_t)J * ldc + I] = val / divisor;
}

// multigrid/transfer.py:38-72 (+ `pressure += correction`, multigrid/solver.py:133-134)
template <typename T>
__global__ void k_prolong(int Hc, int Wc, const T* __restrict__ c, int64_t ldc, int H, int W, Masks m,
                          T* __restrict__ f, int64_t ldf, int accumulate) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= W || j >= H) return;
  T corr = (T)0;
  if (m.fluid(j, i)) {
    double xc = ((double)i + 0.5) * 0.5, yc = ((double)j + 0.5) * 0.5;
    corr = (T)sample_ref(c, ldc, (int64_t)Hc, (int64_t)Wc, xc - 0.5, yc - 0.5);
  }
  int64_t k = (int64_t)j * ldf + i;
  f[k] = accumulate ? f[k] + corr : corr;
}

// multigrid/masks.py:3-27
__global__ void k_coarsen_solid(int Hc, int Wc, const uint8_t* __restrict__ s, int64_t lds, uint8_t* c, int64_t ldc) {
  int I = blockIdx.x * blockDim.x + threadIdx.x;
  int J = blockIdx.y * blockDim.y + threadIdx.y;
  if (I >= Wc || J >= Hc) return;
  const uint8_t* r0 = s + (int64_t)(2 * J) * lds + 2 * I;
  const uint8_t* r1 = r0 + lds;
  c[(int64_t)J * ldc + I] = (r0[0] || r0[1] || r1[0] || r1[1]) ? 1 : 0;
}

}  // namespace sg

using namespace sg;

// ------------------------------------------------------------------ argument checks
// largest grid (bytes of one field) solved by the multi-sweep Jacobi tiles
constexpr int64_t kJacobiTileMaxBytes = (int64_t)8 << 20;

static int check_grid(int64_t H, int64_t W) {
  if (H < 1 || W < 1 || H > (1 << 28) || W > (1 << 28)) return fail(SG_ERR_ARG, "bad grid %lld x %lld", (long long)H, (long long)W);
  return SG_OK;
}

static int check_mask_mode(int mode, const void* a, const void* b) {
  if (mode == SG_MASK_PLANES) {
    if (!a || !b) return fail(SG_ERR_ARG, "mask planes required in SG_MASK_PLANES mode");
    return SG_OK;
  }
  if (mode == SG_MASK_OPEN || mode == SG_MASK_RING) return SG_OK;
  return fail(SG_ERR_ARG, "bad mask mode %d", mode);
}

// Ping-pong buffer of sg_jacobi_solve_noalloc: a fixed array in device memory, so the
// entry point allocates nothing. Host code cannot use the name as a device address;
// its address is looked up once per device with that device current and kept for the
// life of the process (a cudaDeviceReset invalidates it until the library is reloaded).
static __device__ __align__(256) unsigned char g_jacobi_noalloc_scratch[SG_JACOBI_NOALLOC_MAX_BYTES];

static std::mutex g_noalloc_mu;
static void* g_noalloc_addr[256];

static int noalloc_scratch_address(void** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(SG_ERR_CUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
  if (dev < 0 || dev >= 256) return fail(SG_ERR_CAPACITY, "device ordinal %d out of range", dev);
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_jacobi_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return fail(SG_ERR_CUDA, "cudaGetSymbolAddress(static Jacobi scratch): %s", cudaGetErrorString(e));
    g_noalloc_addr[dev] = p;
  }
  *out = g_noalloc_addr[dev];
  return SG_OK;
}

extern "C" {

const char* sg_version(void) { return "smoke_b200 1.0 (sm_100a)"; }
const char* sg_last_error(void) { return last_error_cstr(); }
uint64_t sg_launch_count(void) { return (uint64_t)launch_count(); }

int sg_advect_scalar(int dtype, int64_t H, int64_t W, const void* src, int64_t ld_src, void* dst, int64_t ld_dst,
                     const void* u, int64_t u_rows, int64_t u_cols, int64_t ld_u, const void* v, int64_t v_rows,
                     int64_t v_cols, int64_t ld_v, int mask_mode, const uint8_t* is_fluid, int64_t ld_fluid, double dt,
                     double cell_size, double dissipation, void* stream) {
  SG_CHECK(check_grid(H, W));
  SG_REQUIRE(src && dst && u && v, "null field pointer");
  SG_REQUIRE(u_rows >= 1 && u_cols >= 1 && v_rows >= 1 && v_cols >= 1, "bad velocity shape");
  SG_REQUIRE(ld_src >= W && ld_dst >= W && ld_u >= u_cols && ld_v >= v_cols, "row stride below row length");
  SG_REQUIRE(cell_size > 0.0, "cell_size must be positive");
  SG_REQUIRE(mask_mode != SG_MASK_PLANES || is_fluid, "is_fluid plane required");
  SG_REQUIRE(mask_mode == SG_MASK_PLANES || mask_mode == SG_MASK_OPEN || mask_mode == SG_MASK_RING, "bad mask mode");
  Masks m = make_masks(mask_mode, H, W, nullptr, 0, nullptr, 0, is_fluid, ld_fluid);
  if (mask_mode == SG_MASK_PLANES) m.mode = SG_MASK_PLANES;
  SG_DISPATCH(dtype, {
    SG_MASK_DISPATCH(mask_mode, {
      SG_LAUNCH(k_advect_scalar<T, MM><<<grid2d_rows(W, H), block2d(), 0, as_stream(stream)>>>(
          (int)H, (int)W, (const T*)src, ld_src, (T*)dst, ld_dst, (const T*)u, u_rows, u_cols, ld_u, (const T*)v,
          v_rows, v_cols, ld_v, m.as<MM>(), dt, 1.0 / cell_size, (T)dissipation));
    });
  });
  return check_launch("sg_advect_scalar");
}

int sg_advect_velocity_u(int dtype, int64_t u_rows, int64_t u_cols, const void* u_src, int64_t ld_us, void* u_dst,
                         int64_t ld_ud, const void* v, int64_t v_rows, int64_t v_cols, int64_t ld_v, int mask_mode,
                         const uint8_t* fmu, int64_t ld_fmu, double dt, double cell_size, void* stream) {
  SG_CHECK(check_grid(u_rows, u_cols));
  SG_REQUIRE(u_src && u_dst && v, "null field pointer");
  SG_REQUIRE(ld_us >= u_cols && ld_ud >= u_cols && ld_v >= v_cols && v_rows >= 1 && v_cols >= 1, "bad shape/stride");
  SG_REQUIRE(cell_size > 0.0, "cell_size must be positive");
  SG_CHECK(check_mask_mode(mask_mode, mask_mode == SG_MASK_PLANES ? fmu : (const void*)1, (const void*)1));
  Masks m = make_masks(mask_mode, u_rows, u_cols - 1, fmu, ld_fmu, nullptr, 0, nullptr, 0);
  SG_DISPATCH(dtype, {
    SG_LAUNCH(k_advect_u<T><<<grid2d(u_cols, u_rows), block2d(), 0, as_stream(stream)>>>(
        (int)u_rows, (int)u_cols, (const T*)u_src, ld_us, (T*)u_dst, ld_ud, (const T*)v, v_rows, v_cols, ld_v, m, dt,
        1.0 / cell_size));
  });
  return check_launch("sg_advect_velocity_u");
}

int sg_advect_velocity_v(int dtype, int64_t v_rows, int64_t v_cols, const void* v_src, int64_t ld_vs, void* v_dst,
                         int64_t ld_vd, const void* u, int64_t u_rows, int64_t u_cols, int64_t ld_u, int mask_mode,
                         const uint8_t* fmv, int64_t ld_fmv, double dt, double cell_size, void* stream) {
  SG_CHECK(check_grid(v_rows, v_cols));
  SG_REQUIRE(v_src && v_dst && u, "null field pointer");
  SG_REQUIRE(ld_vs >= v_cols && ld_vd >= v_cols && ld_u >= u_cols && u_rows >= 1 && u_cols >= 1, "bad shape/stride");
  SG_REQUIRE(cell_size > 0.0, "cell_size must be positive");
  SG_CHECK(check_mask_mode(mask_mode, mask_mode == SG_MASK_PLANES ? fmv : (const void*)1, (const void*)1));
  Masks m = make_masks(mask_mode, v_rows - 1, v_cols, nullptr, 0, fmv, ld_fmv, nullptr, 0);
  SG_DISPATCH(dtype, {
    SG_LAUNCH(k_advect_v<T><<<grid2d(v_cols, v_rows), block2d(), 0, as_stream(stream)>>>(
        (int)v_rows, (int)v_cols, (const T*)v_src, ld_vs, (T*)v_dst, ld_vd, (const T*)u, u_rows, u_cols, ld_u, m, dt,
        1.0 / cell_size));
  });
  return check_launch("sg_advect_velocity_v");
}

int sg_advect_velocity(int dtype, int64_t H, int64_t W, const void* u_src, int64_t ld_us, void* u_dst, int64_t ld_ud,
                       const void* v_src, int64_t ld_vs, void* v_dst, int64_t ld_vd, int mask_mode, const uint8_t* fmu,
                       int64_t ld_fmu, const uint8_t* fmv, int64_t ld_fmv, double dt, double cell_size, void* stream) {
  SG_CHECK(check_grid(H, W));
  SG_REQUIRE(u_src && u_dst && v_src && v_dst, "null field pointer");
  SG_REQUIRE(ld_us >= W + 1 && ld_ud >= W + 1 && ld_vs >= W && ld_vd >= W, "row stride below row length");
  SG_REQUIRE(cell_size > 0.0, "cell_size must be positive");
  SG_CHECK(check_mask_mode(mask_mode, fmu, fmv));
  Masks m = make_masks(mask_mode, H, W, fmu, ld_fmu, fmv, ld_fmv, nullptr, 0);
  SG_DISPATCH(dtype, {
    SG_MASK_DISPATCH(mask_mode, {
      SG_LAUNCH(k_advect_uv<T, MM><<<grid2d_rows(W + 1, H + 1), block2d(), 0, as_stream(stream)>>>(
          (int)H, (int)W, (const T*)u_src, ld_us, (T*)u_dst, ld_ud, (const T*)v_src, ld_vs, (T*)v_dst, ld_vd,
          m.as<MM>(), dt, 1.0 / cell_size));
    });
  });
  return check_launch("sg_advect_velocity");
}

int sg_apply_forces(int dtype, int64_t H, int64_t W, void* v, int64_t ld_v, const void* density, int64_t ld_d,
                    const void* temperature, int64_t ld_t, double dt, double gravity, double buoyancy_coefficient,
                    double density_coefficient, double ambient_temperature, int f32_temporaries, void* stream) {
  SG_CHECK(check_grid(H, W));
  SG_REQUIRE(v && density, "null field pointer");
  SG_REQUIRE(ld_v >= W && ld_d >= W && (!temperature || ld_t >= W), "row stride below row length");
  SG_DISPATCH(dtype, {
    SG_LAUNCH(k_apply_forces<T><<<grid2d_rows(W, H + 1), block2d(), 0, as_stream(stream)>>>(
        (int)H, (int)W, (T*)v, ld_v, (const T*)density, ld_d, (const T*)temperature, ld_t, dt, gravity,
        buoyancy_coefficient, density_coefficient, ambient_temperature, f32_temporaries));
  });
  return check_launch("sg_apply_forces");
}

int sg_cool_temperature(int dtype, int64_t H, int64_t W, void* temperature, int64_t ld_t, double ambient,
                        double cooling_rate, double dt, void* stream) {
  SG_CHECK(check_grid(H, W));
  SG_REQUIRE(temperature && ld_t >= W, "bad temperature field");
  double decay = std::exp(-cooling_rate * dt);
  SG_DISPATCH(dtype, {
    SG_LAUNCH(k_cool<T><<<grid2d(W, H), block2d(), 0, as_stream(stream)>>>((int)H, (int)W, (T*)temperature, ld_t, ambient, decay));
  });
  return check_launch("sg_cool_temperature");
}

int sg_compute_divergence(int dtype, int64_t H, int64_t W, const void* u, int64_t ld_u, const void* v, int64_t ld_v,
                          void* div, int64_t ld_div, int mask_mode, const uint8_t* fmu, int64_t ld_fmu,
                          const uint8_t* fmv, int64_t ld_fmv, double cell_size, void* stream) {
  SG_CHECK(check_grid(H, W));
  SG_REQUIRE(u && v && div, "null field pointer");
  SG_REQUIRE(ld_u >= W + 1 && ld_v >= W && ld_div >= W, "row stride below row length");
  SG_REQUIRE(cell_size > 0.0, "cell_size must be positive");
  SG_CHECK(check_mask_mode(mask_mode, fmu, fmv));
  Masks m = make_masks(mask_mode, H, W, fmu, ld_fmu, fmv, ld_fmv, nullptr, 0);
  SG_DISPATCH(dtype, {
    SG_MASK_DISPATCH(mask_mode, {
      SG_LAUNCH(k_divergence<T, MM><<<grid2d_rows(W, H), block2d(), 0, as_stream(stream)>>>(
          (int)H, (int)W, (const T*)u, ld_u, (const T*)v, ld_v, (T*)div, ld_div, m.as<MM>(), 1.0 / cell_size));
    });
  });
  return check_launch("sg_compute_divergence");
}

int sg_compute_residual(int dtype, int64_t H, int64_t W, const void* p, int64_t ld_p, const void* div, int64_t ld_div,
                        int mask_mode, const uint8_t* is_fluid, int64_t ld_fluid, const uint8_t* fmu, int64_t ld_fmu,
                        const uint8_t* fmv, int64_t ld_fmv, double alpha, double reciprocal_beta, void* out,
                        int64_t ld_out, double* sumsq, void* stream) {
  SG_CHECK(check_grid(H, W));
  SG_REQUIRE(p && div && (out || sumsq), "null field pointer");
  SG_REQUIRE(ld_p >= W && ld_div >= W && (!out || ld_out >= W), "row stride below row length");
  SG_REQUIRE(reciprocal_beta != 0.0, "reciprocal_beta must be non-zero");
  SG_CHECK(check_mask_mode(mask_mode, fmu, fmv));
  Masks m = make_masks(mask_mode, H, W, fmu, ld_fmu, fmv, ld_fmv, is_fluid, ld_fluid);
  SG_DISPATCH(dtype, {
    SG_MASK_DISPATCH(mask_mode, {
      SG_LAUNCH(k_residual<T, MM><<<grid2d_rows(W, H), block2d(), 0, as_stream(stream)>>>(
          (int)H, (int)W, (const T*)p, ld_p, (const T*)div, ld_div, m.as<MM>(), alpha, 1.0 / reciprocal_beta, (T*)out,
          ld_out, sumsq));
    });
  });
  return check_launch("sg_compute_residual");
}

int sg_apply_pressure_gradient(int dtype, int64_t H, int64_t W, void* u, int64_t ld_u, void* v, int64_t ld_v,
                               const void* p, int64_t ld_p, int mask_mode, const uint8_t* fmu, int64_t ld_fmu,
                               const uint8_t* fmv, int64_t ld_fmv, double fluid_density, double cell_size, double dt,
                               void* stream) {
  return sg_project(dtype, H, W, u, ld_u, v, ld_v, p, ld_p, mask_mode, fmu, ld_fmu, fmv, ld_fmv, SG_MASK_NONE,
                    nullptr, 0, fluid_density, cell_size, dt, stream);
}

int sg_enforce_boundary_conditions(int dtype, int64_t H, int64_t W, void* u, int64_t ld_u, void* v, int64_t ld_v,
                                   int solid_mode, const uint8_t* solid, int64_t ld_s, void* stream) {
  SG_CHECK(check_grid(H, W));
  SG_REQUIRE(u && v && ld_u >= W + 1 && ld_v >= W, "bad velocity fields");
  SG_REQUIRE(solid_mode == SG_MASK_NONE || solid_mode == SG_MASK_RING || (solid_mode == SG_MASK_PLANES && solid),
             "bad solid mode or missing solid plane");
  if (solid_mode == SG_MASK_NONE) return SG_OK;
  Masks m = make_masks(SG_MASK_OPEN, H, W, nullptr, 0, nullptr, 0, nullptr, 0);
  SG_DISPATCH(dtype, {
    SG_SOLID_DISPATCH(solid_mode, {
      SG_LAUNCH(k_project<T, SG_MASK_OPEN, SM><<<grid2d_rows(W + 1, H + 1), block2d(), 0, as_stream(stream)>>>(
          (int)H, (int)W, (T*)u, ld_u, (T*)v, ld_v, (const T*)nullptr, 0, m.as<SG_MASK_OPEN>(), 0, solid_mode, solid,
          ld_s, 0.0));
    });
  });
  return check_launch("sg_enforce_boundary_conditions");
}

int sg_project(int dtype, int64_t H, int64_t W, void* u, int64_t ld_u, void* v, int64_t ld_v, const void* p,
               int64_t ld_p, int mask_mode, const uint8_t* fmu, int64_t ld_fmu, const uint8_t* fmv, int64_t ld_fmv,
               int solid_mode, const uint8_t* solid, int64_t ld_s, double fluid_density, double cell_size, double dt,
               void* stream) {
  SG_CHECK(check_grid(H, W));
  SG_REQUIRE(u && v && p, "null field pointer");
  SG_REQUIRE(ld_u >= W + 1 && ld_v >= W && ld_p >= W, "row stride below row length");
  SG_REQUIRE(fluid_density != 0.0 && cell_size > 0.0, "bad fluid_density / cell_size");
  SG_CHECK(check_mask_mode(mask_mode, fmu, fmv));
  SG_REQUIRE(solid_mode == SG_MASK_NONE || solid_mode == SG_MASK_RING || (solid_mode == SG_MASK_PLANES && solid),
             "bad solid mode or missing solid plane");
  Masks m = make_masks(mask_mode, H, W, fmu, ld_fmu, fmv, ld_fmv, nullptr, 0);
  double scale = dt / (fluid_density * cell_size);
  SG_DISPATCH(dtype, {
    SG_MASK_DISPATCH(mask_mode, {
      SG_SOLID_DISPATCH(solid_mode, {
        SG_LAUNCH(k_project<T, MM, SM><<<grid2d_rows(W + 1, H + 1), block2d(), 0, as_stream(stream)>>>(
            (int)H, (int)W, (T*)u, ld_u, (T*)v, ld_v, (const T*)p, ld_p, m.as<MM>(), 1, solid_mode, solid, ld_s,
            scale));
      });
    });
  });
  return check_launch("sg_project");
}

int sg_project_metrics(int dtype, int64_t H, int64_t W, const void* u_in, int64_t ld_ui, const void* v_in,
                       int64_t ld_vi, void* u_out, int64_t ld_uo, void* v_out, int64_t ld_vo, const void* p,
                       int64_t ld_p, int mask_mode, const uint8_t* fmu, int64_t ld_fmu, const uint8_t* fmv,
                       int64_t ld_fmv, const uint8_t* is_fluid, int64_t ld_fluid, int solid_mode, const uint8_t* solid,
                       int64_t ld_s, double fluid_density, double cell_size, double dt, double alpha,
                       double reciprocal_beta, void* div, int64_t ld_div, void* res, int64_t ld_res, void* stream) {
  SG_CHECK(check_grid(H, W));
  SG_REQUIRE(u_in && v_in && u_out && v_out && p && div && res, "null field pointer");
  SG_REQUIRE(u_in != u_out && v_in != v_out, "the projection here is out of place");
  SG_REQUIRE(ld_ui >= W + 1 && ld_vi >= W && ld_uo >= W + 1 && ld_vo >= W && ld_p >= W && ld_div >= W && ld_res >= W,
             "row stride below row length");
  SG_REQUIRE(fluid_density != 0.0 && cell_size > 0.0 && reciprocal_beta != 0.0, "bad coefficients");
  SG_CHECK(check_mask_mode(mask_mode, fmu, fmv));
  SG_REQUIRE(mask_mode != SG_MASK_PLANES || is_fluid, "is_fluid plane required");
  SG_REQUIRE(solid_mode == SG_MASK_NONE || solid_mode == SG_MASK_RING || (solid_mode == SG_MASK_PLANES && solid),
             "bad solid mode or missing solid plane");
  Masks m = make_masks(mask_mode, H, W, fmu, ld_fmu, fmv, ld_fmv, is_fluid, ld_fluid);
  const double scale = dt / (fluid_density * cell_size);
  SG_DISPATCH(dtype, {
    SG_MASK_DISPATCH(mask_mode, {
      SG_SOLID_DISPATCH(solid_mode, {
        SG_LAUNCH(k_project_metrics<T, MM, SM><<<dim3((unsigned)((W + 1 + kBX - 1) / kBX),
                                                       (unsigned)((H + kBY * kTailRows - 1) / (kBY * kTailRows))),
                                                  block2d(), 0, as_stream(stream)>>>(
            (int)H, (int)W, (const T*)u_in, ld_ui, (const T*)v_in, ld_vi, (T*)u_out, ld_uo, (T*)v_out, ld_vo,
            (const T*)p, ld_p, m.as<MM>(), solid_mode, solid, ld_s, scale, (T*)div, ld_div, 1.0 / cell_size, alpha,
            1.0 / reciprocal_beta, (T*)res, ld_res));
      });
    });
  });
  return check_launch("sg_project_metrics");
}

int sg_emit_scalar(int dtype, int64_t H, int64_t W, void* field, int64_t ld, double value, double dt, double pos_x,
                   double pos_y, double radius, int approach, void* stream) {
  SG_CHECK(check_grid(H, W));
  SG_REQUIRE(field && ld >= W, "bad field");
  SG_REQUIRE(approach >= 0 && approach <= 3, "approach must be 0..3");
  // emitters.py:52-56: bounding box with Python int() truncation.
  int64_t x_min = (int64_t)(pos_x - radius - 1.0), x_max = (int64_t)(pos_x + radius + 2.0);
  int64_t y_min = (int64_t)(pos_y - radius - 1.0), y_max = (int64_t)(pos_y + radius + 2.0);
  if (x_min < 0) x_min = 0;
  if (y_min < 0) y_min = 0;
  if (x_max > W) x_max = W;
  if (y_max > H) y_max = H;
  if (x_max <= x_min || y_max <= y_min) return SG_OK;
  int64_t bw = x_max - x_min, bh = y_max - y_min;
  SG_DISPATCH(dtype, {
    SG_LAUNCH(k_emit<T><<<grid2d(bw, bh), block2d(), 0, as_stream(stream)>>>((int)bw, (int)bh, (int)x_min, (int)y_min, (T*)field,
                                                                   ld, value, dt, pos_x, pos_y, radius, approach));
  });
  return check_launch("sg_emit_scalar");
}

int sg_plume_sources(int dtype, int64_t H, int64_t W, void* density, int64_t ld_d, void* u, int64_t ld_u, void* v,
                     int64_t ld_v, int n_sources, const double* sources, uint64_t seed, int64_t step, void* stream) {
  SG_CHECK(check_grid(H, W));
  SG_REQUIRE(density && u && v && ld_d >= W && ld_u >= W + 1 && ld_v >= W, "bad fields");
  SG_REQUIRE(n_sources >= 0 && n_sources <= kMaxPlumes && (n_sources == 0 || sources),
             "source table must hold 0..%d rows", kMaxPlumes);
  if (n_sources == 0) return SG_OK;
  PlumeTable tab;
  std::memset(&tab, 0, sizeof(tab));
  tab.n = n_sources;
  // union of the sources' boxes: every cell centre / face strictly inside a disc lies in
  // [cx - r - 1, cx + r + 1] x [cy - r - 1, cy + r + 1]
  double xlo = 1e300, xhi = -1e300, ylo = 1e300, yhi = -1e300;
  for (int s = 0; s < n_sources; ++s) {
    const double* q = sources + 6 * s;
    SG_REQUIRE(std::isfinite(q[0]) && std::isfinite(q[1]) && std::isfinite(q[2]) && q[2] >= 0.0,
               "source %d: centre and radius must be finite, radius >= 0", s);
    for (int k = 0; k < 6; ++k) tab.row[6 * s + k] = q[k];
    xlo = std::min(xlo, q[0] - q[2] - 1.0);
    xhi = std::max(xhi, q[0] + q[2] + 1.0);
    ylo = std::min(ylo, q[1] - q[2] - 1.0);
    yhi = std::max(yhi, q[1] + q[2] + 1.0);
  }
  int64_t x0 = std::max<int64_t>(0, (int64_t)std::floor(std::max(xlo, -1.0)));
  int64_t y0 = std::max<int64_t>(0, (int64_t)std::floor(std::max(ylo, -1.0)));
  int64_t x1 = std::min<int64_t>(W, (int64_t)std::ceil(std::min(xhi, (double)W + 1.0)));
  int64_t y1 = std::min<int64_t>(H, (int64_t)std::ceil(std::min(yhi, (double)H + 1.0)));
  if (x1 < x0 || y1 < y0) return SG_OK;
  tab.x0 = (int)x0;
  tab.y0 = (int)y0;
  SG_DISPATCH(dtype, {
    SG_LAUNCH(k_plume<T><<<grid2d(x1 - x0 + 1, y1 - y0 + 1), block2d(), 0, as_stream(stream)>>>(
        (int)H, (int)W, (T*)density, ld_d, (T*)u, ld_u, (T*)v, ld_v, tab, seed, step));
  });
  return check_launch("sg_plume_sources");
}

int sg_build_masks(int64_t H, int64_t W, const uint8_t* solid, int64_t ld_s, uint8_t* fmu, int64_t ld_fmu, uint8_t* fmv,
                   int64_t ld_fmv, uint8_t* is_fluid, int64_t ld_fluid, void* stream) {
  SG_CHECK(check_grid(H, W));
  SG_REQUIRE(solid && ld_s >= W, "bad solid plane");
  SG_LAUNCH(k_build_masks<<<grid2d(W + 1, H + 1), block2d(), 0, as_stream(stream)>>>((int)H, (int)W, solid, ld_s, fmu, ld_fmu, fmv,
                                                                          ld_fmv, is_fluid, ld_fluid));
  return check_launch("sg_build_masks");
}

int sg_jacobi_solve(int dtype, int64_t H, int64_t W, void* p, int64_t ld_p, const void* div, int64_t ld_div,
                    int mask_mode, const uint8_t* fmu, int64_t ld_fmu, const uint8_t* fmv, int64_t ld_fmv, double alpha,
                    double reciprocal_beta, int iterations, void* scratch, void* stream) {
  SG_CHECK(check_grid(H, W));
  SG_REQUIRE(p && div && scratch, "null pointer (p, div and scratch are required)");
  SG_REQUIRE(ld_p >= W && ld_div >= W, "row stride below row length");
  SG_REQUIRE(iterations >= 0, "iterations must be >= 0");
  SG_CHECK(check_mask_mode(mask_mode, fmu, fmv));
  Masks m = make_masks(mask_mode, H, W, fmu, ld_fmu, fmv, ld_fmv, nullptr, 0);
  cudaStream_t s = as_stream(stream);
  SG_DISPATCH(dtype, {
    T* a = (T*)p;
    int64_t lda = ld_p;
    T* b = (T*)scratch;
    int64_t ldb = W;
    // grids that sit in L2: kJG sweeps per launch on shared-memory tiles (same iterates)
    const bool tiles = H * W * (int64_t)sizeof(T) <= kJacobiTileMaxBytes;
    const int per = tiles ? kJG : 1;
    for (int it = 0; it < iterations; it += per) {
      if (tiles) {
        const int n = iterations - it < kJG ? iterations - it : kJG;
        SG_MASK_DISPATCH(mask_mode, {
          SG_LAUNCH(k_jacobi_tiles<T, MM><<<dim3((unsigned)((W + kJTC - 1) / kJTC), (unsigned)((H + kJTR - 1) / kJTR)),
                                           kJT, 0, s>>>((int)H, (int)W, a, lda, b, ldb, (const T*)div, ld_div,
                                                        m.as<MM>(), alpha, reciprocal_beta, n));
        });
        T* t = a;
        a = b;
        b = t;
        int64_t tl = lda;
        lda = ldb;
        ldb = tl;
        continue;
      }
      SG_LAUNCH(k_jacobi<T><<<grid2d(W, H), block2d(), 0, s>>>((int)H, (int)W, a, lda, b, ldb, (const T*)div, ld_div, m, alpha,
                                                     reciprocal_beta));
      T* t = a;
      a = b;
      b = t;
      int64_t tl = lda;
      lda = ldb;
      ldb = tl;
    }
    SG_CHECK(check_launch("sg_jacobi_solve"));
    if (a != (T*)p) {
      cudaError_t e = cudaMemcpy2DAsync(p, ld_p * sizeof(T), a, lda * sizeof(T), W * sizeof(T), H,
                                        cudaMemcpyDeviceToDevice, s);
      if (e != cudaSuccess) return fail(SG_ERR_CUDA, "sg_jacobi_solve copy-back: %s", cudaGetErrorString(e));
    }
  });
  return SG_OK;
}

int sg_jacobi_solve_noalloc(int dtype, int64_t H, int64_t W, void* p, int64_t ld_p, const void* div, int64_t ld_div,
                            int mask_mode, const uint8_t* fmu, int64_t ld_fmu, const uint8_t* fmv, int64_t ld_fmv,
                            double alpha, double reciprocal_beta, int iterations, void* stream) {
  SG_CHECK(check_grid(H, W));
  int64_t elem = dtype == SG_F32 ? 4 : (dtype == SG_F64 ? 8 : 0);
  if (elem == 0) return fail(SG_ERR_DTYPE, "unsupported dtype code %d", dtype);
  if (H * W * elem > (int64_t)SG_JACOBI_NOALLOC_MAX_BYTES)
    return fail(SG_ERR_CAPACITY, "sg_jacobi_solve_noalloc: %lld x %lld cells of %lld bytes exceed the %u-byte static "
                "scratch; use sg_jacobi_solve with a caller buffer", (long long)H, (long long)W, (long long)elem,
                (unsigned)SG_JACOBI_NOALLOC_MAX_BYTES);
  void* scratch = nullptr;
  SG_CHECK(noalloc_scratch_address(&scratch));
  return sg_jacobi_solve(dtype, H, W, p, ld_p, div, ld_div, mask_mode, fmu, ld_fmu, fmv, ld_fmv, alpha,
                         reciprocal_beta, iterations, scratch, stream);
}

int sg_rbsor_solve(int dtype, int64_t H, int64_t W, void* p, int64_t ld_p, const void* div, int64_t ld_div,
                   int mask_mode, const uint8_t* fmu, int64_t ld_fmu, const uint8_t* fmv, int64_t ld_fmv, double alpha,
                   double reciprocal_beta, double omega, int iterations, void* stream) {
  SG_CHECK(check_grid(H, W));
  SG_REQUIRE(p && div && ld_p >= W && ld_div >= W, "bad fields");
  SG_REQUIRE(iterations >= 0, "iterations must be >= 0");
  SG_CHECK(check_mask_mode(mask_mode, fmu, fmv));
  Masks m = make_masks(mask_mode, H, W, fmu, ld_fmu, fmv, ld_fmv, nullptr, 0);
  cudaStream_t s = as_stream(stream);
  dim3 g = grid2d((W + 1) / 2, H);
  SG_DISPATCH(dtype, {
    for (int it = 0; it < iterations; ++it)
      for (int color = 0; color < 2; ++color)
        SG_LAUNCH(k_rbsor_half<T><<<g, block2d(), 0, s>>>((int)H, (int)W, (T*)p, ld_p, (const T*)div, ld_div, m, alpha,
                                                 reciprocal_beta, omega, color));
  });
  return check_launch("sg_rbsor_solve");
}

int sg_gauss_seidel_solve(int dtype, int64_t H, int64_t W, void* p, int64_t ld_p, const void* div, int64_t ld_div,
                          int mask_mode, const uint8_t* fmu, int64_t ld_fmu, const uint8_t* fmv, int64_t ld_fmv,
                          double alpha, double reciprocal_beta, int iterations, void* stream) {
  SG_CHECK(check_grid(H, W));
  SG_REQUIRE(p && div && ld_p >= W && ld_div >= W, "bad fields");
  SG_REQUIRE(iterations >= 0, "iterations must be >= 0");
  SG_CHECK(check_mask_mode(mask_mode, fmu, fmv));
  if (iterations == 0) return SG_OK;
  Masks m = make_masks(mask_mode, H, W, fmu, ld_fmu, fmv, ld_fmv, nullptr, 0);
  SG_DISPATCH(dtype, {
    SG_LAUNCH(k_gauss_seidel<T><<<1, 1024, 0, as_stream(stream)>>>((int)H, (int)W, (T*)p, ld_p, (const T*)div, ld_div, m, alpha,
                                                         reciprocal_beta, iterations));
  });
  return check_launch("sg_gauss_seidel_solve");
}

int sg_mg_restrict_average(int dtype, int64_t H, int64_t W, const void* fine, int64_t ld_f, int mask_mode,
                           const uint8_t* is_fluid, int64_t ld_fluid, void* coarse, int64_t ld_c, int64_t Hc, int64_t Wc,
                           double divisor, void* stream) {
  SG_CHECK(check_grid(H, W));
  SG_REQUIRE(fine && coarse && ld_f >= W && ld_c >= Wc, "bad fields");
  SG_REQUIRE(Hc >= 1 && Wc >= 1 && 2 * Hc <= H && 2 * Wc <= W, "coarse grid must be at most half the fine grid");
  SG_REQUIRE(mask_mode != SG_MASK_PLANES || is_fluid, "is_fluid plane required");
  SG_REQUIRE(mask_mode == SG_MASK_PLANES || mask_mode == SG_MASK_OPEN || mask_mode == SG_MASK_RING, "bad mask mode");
  SG_REQUIRE(divisor != 0.0, "divisor must be non-zero");
  Masks m = make_masks(mask_mode, H, W, nullptr, 0, nullptr, 0, is_fluid, ld_fluid);
  SG_DISPATCH(dtype, {
    SG_LAUNCH(k_restrict_avg<T><<<grid2d(Wc, Hc), block2d(), 0, as_stream(stream)>>>((int)H, (int)W, (const T*)fine, ld_f, m,
                                                                            (T*)coarse, ld_c, (int)Hc, (int)Wc,
                                                                            (T)divisor));
  });
  return check_launch("sg_mg_restrict_average");
}

int sg_mg_prolong(int dtype, int64_t Hc, int64_t Wc, const void* coarse, int64_t ld_c, int64_t H, int64_t W, int mask_mode,
                  const uint8_t* is_fluid, int64_t ld_fluid, void* fine, int64_t ld_f, int accumulate, void* stream) {
  SG_CHECK(check_grid(H, W));
  SG_CHECK(check_grid(Hc, Wc));
  SG_REQUIRE(fine && coarse && ld_f >= W && ld_c >= Wc, "bad fields");
  SG_REQUIRE(mask_mode != SG_MASK_PLANES || is_fluid, "is_fluid plane required");
  SG_REQUIRE(mask_mode == SG_MASK_PLANES || mask_mode == SG_MASK_OPEN || mask_mode == SG_MASK_RING, "bad mask mode");
  Masks m = make_masks(mask_mode, H, W, nullptr, 0, nullptr, 0, is_fluid, ld_fluid);
  SG_DISPATCH(dtype, {
    SG_LAUNCH(k_prolong<T><<<grid2d(W, H), block2d(), 0, as_stream(stream)>>>((int)Hc, (int)Wc, (const T*)coarse, ld_c, (int)H,
                                                                     (int)W, m, (T*)fine, ld_f, accumulate));
  });
  return check_launch("sg_mg_prolong");
}

int sg_mg_coarsen_solid(int64_t H, int64_t W, const uint8_t* solid, int64_t ld_s, uint8_t* coarse, int64_t ld_c,
                        void* stream) {
  SG_CHECK(check_grid(H, W));
  SG_REQUIRE(solid && coarse && ld_s >= W, "bad planes");
  int64_t Hc = H / 2, Wc = W / 2;
  if (Hc < 1 || Wc < 1) return SG_OK;
  SG_REQUIRE(ld_c >= Wc, "bad coarse stride");
  SG_LAUNCH(k_coarsen_solid<<<grid2d(Wc, Hc), block2d(), 0, as_stream(stream)>>>((int)Hc, (int)Wc, solid, ld_s, coarse, ld_c));
  return check_launch("sg_mg_coarsen_solid");
}

}  // extern "C"

SG_BOUNDS_ACCESSOR(operators)

extern "C" {
int sg_bounds_line_gmg(unsigned* line, int clear);
int sg_bounds_line_batch(unsigned* line, int clear);
int sg_bounds_line_rbsor_split(unsigned* line, int clear);
int sg_bounds_line_advect_fast(unsigned* line, int clear);
int sg_bounds_line_adjoint(unsigned* line, int clear);
int sg_bounds_line_metrics(unsigned* line, int clear);

int sg_bounds_check_enabled(void) { return SG_BOUNDS_CHECK; }

int sg_bounds_check(unsigned* first_line, int* unit, int clear) {
  SG_REQUIRE(first_line && unit, "null output");
  int (*const fns[])(unsigned*, int) = {sg_bounds_line_operators,   sg_bounds_line_gmg,     sg_bounds_line_batch,
                                        sg_bounds_line_rbsor_split, sg_bounds_line_advect_fast,
                                        sg_bounds_line_adjoint,     sg_bounds_line_metrics};
  *first_line = 0;
  *unit = -1;
  for (int k = 0; k < (int)(sizeof(fns) / sizeof(fns[0])); ++k) {
    unsigned line = 0;
    const int rc = fns[k](&line, clear);
    if (rc != SG_OK) return fail(rc, "bounds-check word of unit %d unreadable", k);
    if (line && !*first_line) {
      *first_line = line;
      *unit = k;
    }
  }
  return SG_OK;
}
}  // extern "C"
