// Batched smoke steps: many independent scenes of uneven grid sizes advance together.
//
// Every scene is the default scene of SmokeSimulation2D (open-box kernel masks, a solid
// ring zeroed by the boundary step) in float32 with one overwriting plume source and its
// own buoyancy coefficient, cell size and time step. All scenes' fields live in shared
// pools (one per field kind, scene by scene, row stride = row length). Each operator of the
// step is ONE persistent launch over a work list of tiles (scene, tile row, tile column):
// one resident wave of 256-thread blocks strides over the list, each tile being TX x TY
// cells of one scene, so small and large scenes fill the GPU together. The per-cell arithmetic is the single-grid
// operators' own (cell_ops.cuh); this unit is compiled with -fmad=false like theirs.
//
// The pressure solve is the convergent multigrid of the single-grid solver (red-black
// Gauss-Seidel with omega, full-weighting restriction, bilinear prolongation, exact solve
// on the coarsest level <= 8 x 8 through its pseudo-inverse; each side of a level is one
// launch over a tile list of all scenes: the single-grid register-tile bodies of
// gmg_regtile.cuh on depths 0-3, the shared-memory 16 x 16 tile bodies of gmg_tiled.cuh
// below, sweeps, residual and restriction on chip) in the single-grid solver's
// mixed precision: float32 cycles on the correction equation inside float64 iterative
// refinement (p and the residual b - A p in float64), until each scene's relative residual
// ||b - A p|| / ||b|| is <= tol; the pressure the projection uses is p rounded to float32.
// (Cycling a float32 p directly stalls near 1e-6 on 256^2 scenes.) The scenes'
// hierarchies have different depths; one cycle is a single schedule over depths (V or W,
// the W recursion repeated only where some scene goes deeper) in which a launch at depth
// k touches the scenes that have a level k (the coarse solve: the scenes whose coarsest
// level is k; re-solving a coarsest level is idempotent, so the shared W schedule gives
// every scene its own W-cycle). Scenes that reached the tolerance drop out of the launches;
// the cycle loop is the WHILE node of a CUDA graph that captures the whole step.
//
// A project-written autotuner times the step for every combination of tile shape, sweeps
// per level and cycle type on a copy of the state and keeps the fastest.

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "cell_ops.cuh"

namespace sg {

bool open_box_pinv(int H, int W, std::vector<double>& out);

#include "gmg_weights.cuh"
#include "gmg_tiled.cuh"
#define SG_REGTILE_BODIES_ONLY
#include "gmg_regtile.cuh"
#undef SG_REGTILE_BODIES_ONLY

constexpr int kBMaxLev = 12;
constexpr int kBThreads = 256;

struct BScene {
  int H, W, nlev, pad;
  double inv, dt, alpha, scale, gravity, dcoef;  // 1/h, dt, -h^2 rho / dt, dt / (rho h), g, buoyancy coefficient
  double src[6];                                 // plume row (cx, cy, r, density, v, noise) in cells
  int64_t oc, ou, ov;                            // element offsets in the cell / u-face / v-face pools
  int64_t olev[kBMaxLev];                        // level k >= 1: element offset in the level pools
  int lH[kBMaxLev], lW[kBMaxLev];
  int64_t opinv;                                 // coarsest pseudo-inverse in the pinv pool
};

struct BTile {
  int scene;
  short ty, tx;
};

struct BPools {
  float* d[2];
  float* u[2];
  float* v[2];
  float *div, *p, *b0, *res, *e, *b;  // p: the float32 pressure, and the cycles' fine correction
  float *e2c, *e2l;                     // pre-smoothed corrections: fine level (cell pool), levels >= 1
  float* b1;                            // the fine rhs of odd cycles (b0: even cycles)
  double* r64;                          // the fine residual alpha div - A p64, carried in float64
  double* p64;                          // the float64 pressure of the refinement
  const double* pinv;
  const BScene* scenes;
  double *bn2, *rn2, *relres;
  int *active, *cycles;
  long long* total_cycles;
};

// The cycle schedule state in device memory.
struct BCtl {
  double tol;
  int max_cycles, n_scenes, any, steps;
  long long loops;  // cycle-loop iterations run since bind (all scenes together)
};

__device__ __forceinline__ MasksT<SG_MASK_OPEN> open_masks(int H, int W) {
  MasksT<SG_MASK_OPEN> m;
  m.fmu = m.fmv = m.fl = nullptr;
  m.ldu = m.ldv = m.ldf = 0;
  m.mode = SG_MASK_OPEN;
  m.H = H;
  m.W = W;
  return m;
}

__device__ __forceinline__ float b_rcp(int n) {
  return n == 4 ? 0.25f : (n == 3 ? (float)(1.0 / 3.0) : (n == 2 ? 0.5f : 1.0f));
}

// full-weighting weight of fine index i towards coarse index I (n coarse cells), the
// transpose of the clamped bilinear prolongation
__device__ __forceinline__ float b_w1(int i, int I, int n) {
  int h = i >> 1;
  int x = h + ((i & 1) ? 1 : -1);
  x = x < 0 ? 0 : (x > n - 1 ? n - 1 : x);
  return (h == I ? 0.75f : 0.0f) + (x == I ? 0.25f : 0.0f);
}

// Level k of a scene: e and b arrays (level 0: p and the rhs) with their shape.
struct BLevel {
  float* e;
  float* b;
  int H, W;
};

__device__ __forceinline__ BLevel level_of(const BPools& P, const BScene& s, int k) {
  BLevel L;
  if (k == 0) {
    L.e = P.p + s.oc;
    L.b = P.b0 + s.oc;
    L.H = s.H;
    L.W = s.W;
  } else {
    L.e = P.e + s.olev[k];
    L.b = P.b + s.olev[k];
    L.H = s.lH[k];
    L.W = s.lW[k];
  }
  return L;
}

// The pre-smoothed correction of level k (the fused level kernels' second buffer).
__device__ __forceinline__ float* e2_of(const BPools& P, const BScene& s, int k) {
  return k == 0 ? P.e2c + s.oc : P.e2l + s.olev[k];
}

__device__ __forceinline__ float b_residual(const BLevel& L, int j, int i) {
  const int o = j * L.W + i;
  const float x = L.e[o];
  float acc = L.b[o];
  if (i > 0) acc += L.e[o - 1] - x;
  if (i < L.W - 1) acc += L.e[o + 1] - x;
  if (j > 0) acc += L.e[o - L.W] - x;
  if (j < L.H - 1) acc += L.e[o + L.W] - x;
  return acc;
}

// -------------------------------------------------------------- persistent tile loop
template <int TX, int TY, class F>
__device__ __forceinline__ void for_tiles(const BTile* __restrict__ work, int n, const F& f) {
  const int lx = threadIdx.x % TX, ly = threadIdx.x / TX;
  for (int w = blockIdx.x; w < n; w += gridDim.x) {
    const BTile t = work[w];
    f(t.scene, (int)t.ty * TY + ly, (int)t.tx * TX + lx);
  }
}

// Same, with one double per thread reduced over the tile's block and added to out[scene].
template <int TX, int TY, class F>
__device__ __forceinline__ void for_tiles_sum(const BTile* __restrict__ work, int n, double* out, const F& f) {
  const int lx = threadIdx.x % TX, ly = threadIdx.x / TX;
  for (int w = blockIdx.x; w < n; w += gridDim.x) {
    const BTile t = work[w];
    const double v = f(t.scene, (int)t.ty * TY + ly, (int)t.tx * TX + lx);
    const double s = block_sum(v);
    if (threadIdx.x == 0 && s != 0.0) atomicAdd(out + t.scene, s);
  }
}

// -------------------------------------------------------------- step operators
// Velocity buffers: the state lives in u/v[kVel] between steps; u/v[kVelAdv] holds the
// advected (and forced) velocity until the projection writes the projected one back into
// u/v[kVel]. Density ping-pongs between d[0] and d[1] by the step's parity.
constexpr int kVel = 0, kVelAdv = 1;

// Batched sources carry no noise (amplitude 0), so the step index the noise would hash is
// not needed and the captured step graph can be replayed as is.
struct OpPlume {
  BPools P;
  int cur;
  uint64_t seed;
  int64_t step;
  __device__ void operator()(int sc, int j, int i) const {
    const BScene& s = P.scenes[sc];
    if (j > s.H || i > s.W) return;
    plume_point(j, i, s.H, s.W, P.d[cur] + s.oc, (int64_t)s.W, P.u[kVel] + s.ou, (int64_t)s.W + 1, P.v[kVel] + s.ov,
                (int64_t)s.W, s.src, 1, seed + (uint64_t)sc, step);
  }
};

struct OpForces {
  BPools P;
  int cur;
  __device__ void operator()(int sc, int j, int i) const {
    const BScene& s = P.scenes[sc];
    if (j > s.H || i >= s.W) return;
    forces_face(j, i, s.H, s.W, P.v[kVel] + s.ov, (int64_t)s.W, (const float*)(P.d[cur] + s.oc), (int64_t)s.W,
                (const float*)nullptr, 0, s.dt, s.gravity, 0.0, s.dcoef, 0.0, 1);
  }
};

struct OpAdvectUV {
  BPools P;
  __device__ void operator()(int sc, int j, int i) const {
    const BScene& s = P.scenes[sc];
    const int H = s.H, W = s.W;
    const MasksT<SG_MASK_OPEN> m = open_masks(H, W);
    const float* us = P.u[kVel] + s.ou;
    const float* vs = P.v[kVel] + s.ov;
    if (j < H && i <= W)
      P.u[kVelAdv][s.ou + (int64_t)j * (W + 1) + i] =
          m.u(j, i) ? advect_u_face(j, i, us, (int64_t)W + 1, (int64_t)H, (int64_t)W + 1, vs, (int64_t)H + 1,
                                    (int64_t)W, (int64_t)W, s.dt, s.inv)
                    : 0.0f;
    if (j <= H && i < W)
      P.v[kVelAdv][s.ov + (int64_t)j * W + i] =
          m.v(j, i) ? advect_v_face(j, i, vs, (int64_t)W, (int64_t)H + 1, (int64_t)W, us, (int64_t)H, (int64_t)W + 1,
                                    (int64_t)W + 1, s.dt, s.inv)
                    : 0.0f;
  }
};

struct OpAdvectD {
  BPools P;
  int cur;
  float diss;
  __device__ void operator()(int sc, int j, int i) const {
    const BScene& s = P.scenes[sc];
    const int H = s.H, W = s.W;
    if (j >= H || i >= W) return;
    const MasksT<SG_MASK_OPEN> m = open_masks(H, W);
    P.d[1 - cur][s.oc + (int64_t)j * W + i] =
        advect_scalar_cell(j, i, H, W, (const float*)(P.d[cur] + s.oc), (int64_t)W,
                           (const float*)(P.u[kVelAdv] + s.ou), (int64_t)H, (int64_t)W + 1, (int64_t)W + 1,
                           (const float*)(P.v[kVelAdv] + s.ov), (int64_t)H + 1, (int64_t)W, (int64_t)W, m, s.dt,
                           s.inv, diss);
  }
};

// The end of the step on one cell tile list (simulation.py:245-265): the pressure out of the
// float64 solve, the gradient subtraction with the wall conditions written out of place into
// the velocity state (each thread projects its cell's four faces from the advected velocity
// and stores the lower and left ones, the last column and row also the outer ones), the
// divergence of the projected faces and the reference residual of the pressure.
struct OpTail {
  BPools P;
  __device__ void operator()(int sc, int j, int i) const {
    const BScene& s = P.scenes[sc];
    const int H = s.H, W = s.W;
    if (j >= H || i >= W) return;
    using MK = MasksT<SG_MASK_OPEN>;
    const MK m = open_masks(H, W);
    const double* q = P.p64 + s.oc + (int64_t)j * W + i;
    const float c = (float)q[0];
    const float pl = i > 0 ? (float)q[-1] : c, pr = i < W - 1 ? (float)q[1] : c;
    const float pd = j > 0 ? (float)q[-W] : c, pu = j < H - 1 ? (float)q[W] : c;
    const float* ua = P.u[kVelAdv] + s.ou + (int64_t)j * (W + 1) + i;
    const float* va = P.v[kVelAdv] + s.ov + (int64_t)j * W + i;
    const float ul = projected_u_pv<float, MK, SG_MASK_RING>(j, i, H, W, ua[0], c, pl, m, SG_MASK_RING, nullptr, 0,
                                                           s.scale);
    const float ur = projected_u_pv<float, MK, SG_MASK_RING>(j, i + 1, H, W, ua[1], pr, c, m, SG_MASK_RING, nullptr,
                                                           0, s.scale);
    const float vd = projected_v_pv<float, MK, SG_MASK_RING>(j, i, H, W, va[0], c, pd, m, SG_MASK_RING, nullptr, 0,
                                                           s.scale);
    const float vu = projected_v_pv<float, MK, SG_MASK_RING>(j + 1, i, H, W, va[W], pu, c, m, SG_MASK_RING, nullptr,
                                                           0, s.scale);
    float* u = P.u[kVel] + s.ou + (int64_t)j * (W + 1) + i;
    float* v = P.v[kVel] + s.ov + (int64_t)j * W + i;
    u[0] = ul;
    if (i == W - 1) u[1] = ur;
    v[0] = vd;
    if (j == H - 1) v[W] = vu;
    const int64_t o = s.oc + (int64_t)j * W + i;
    const float dv = divergence_from_faces(j, i, ul, ur, vd, vu, m, s.inv);
    P.p[o] = c;
    P.div[o] = dv;
    P.res[o] = residual_from_values(j, i, H, W, c, pl, pr, pd, pu, dv, m, s.alpha, 4.0);
  }
};

// -------------------------------------------------------------- solver operators
// The divergence of the advected velocity and b = alpha div: the first cycle's rhs (the
// residual of p = 0) in float32 and float64, p64 = 0, ||b||^2 per scene. With depth 0 on
// the tile-list kernels (tiles0), p is that depth's correction (zeroed here) and div feeds
// the fine residual (stored here).
struct OpRhs {
  BPools P;
  int tiles0;
  __device__ double operator()(int sc, int j, int i) const {
    const BScene& s = P.scenes[sc];
    if (j >= s.H || i >= s.W) return 0.0;
    const MasksT<SG_MASK_OPEN> m = open_masks(s.H, s.W);
    const float dv = divergence_cell(j, i, (const float*)(P.u[kVelAdv] + s.ou), (int64_t)s.W + 1,
                                     (const float*)(P.v[kVelAdv] + s.ov), (int64_t)s.W, m, s.inv);
    const int64_t o = s.oc + (int64_t)j * s.W + i;
    const double b = s.alpha * (double)dv;
    P.b0[o] = (float)b;
    P.r64[o] = b;
    P.p64[o] = 0.0;
    if (tiles0) {
      P.div[o] = dv;
      P.p[o] = 0.0f;
    }
    return b * b;
  }
};

// p64 += the cycle's correction, which restarts from 0.
struct OpCorrect {
  BPools P;
  __device__ void operator()(int sc, int j, int i) const {
    if (!P.active[sc]) return;
    const BScene& s = P.scenes[sc];
    if (j >= s.H || i >= s.W) return;
    const int64_t o = s.oc + (int64_t)j * s.W + i;
    P.p64[o] += (double)P.p[o];
    P.p[o] = 0.0f;
  }
};

struct OpRelax {
  BPools P;
  int k, colour;
  float omega;
  __device__ void operator()(int sc, int j, int i) const {
    if (!P.active[sc]) return;
    const BScene& s = P.scenes[sc];
    if (k >= s.nlev - 1) return;
    const BLevel L = level_of(P, s, k);
    if (j >= L.H || i >= L.W || ((i + j) & 1) != colour) return;
    const int o = j * L.W + i;
    float acc = L.b[o];
    int n = 0;
    if (i > 0) { acc += L.e[o - 1]; ++n; }
    if (i < L.W - 1) { acc += L.e[o + 1]; ++n; }
    if (j > 0) { acc += L.e[o - L.W]; ++n; }
    if (j < L.H - 1) { acc += L.e[o + L.W]; ++n; }
    if (n == 0) return;
    const float x = L.e[o];
    L.e[o] = x + omega * (acc * b_rcp(n) - x);
  }
};

// level k + 1 (coarse cell (J, I)): b = P^T (b - A e) of level k, e = 0
struct OpRestrict {
  BPools P;
  int k;
  __device__ void operator()(int sc, int J, int I) const {
    if (!P.active[sc]) return;
    const BScene& s = P.scenes[sc];
    if (k >= s.nlev - 1) return;
    const BLevel F = level_of(P, s, k);
    const BLevel C = level_of(P, s, k + 1);
    if (J >= C.H || I >= C.W) return;
    float acc = 0.0f;
#pragma unroll
    for (int dj = 0; dj < 4; ++dj) {
      const int j = 2 * J - 1 + dj;
      if (j < 0 || j >= F.H) continue;
      const float wy = b_w1(j, J, C.H);
      if (wy == 0.0f) continue;
#pragma unroll
      for (int di = 0; di < 4; ++di) {
        const int i = 2 * I - 1 + di;
        if (i < 0 || i >= F.W) continue;
        const float w = wy * b_w1(i, I, C.W);
        if (w != 0.0f) acc += w * b_residual(F, j, i);
      }
    }
    C.b[J * C.W + I] = acc;
    C.e[J * C.W + I] = 0.0f;
  }
};

// level k: e += P e(k + 1), bilinear with clamped candidates
struct OpProlong {
  BPools P;
  int k;
  __device__ void operator()(int sc, int j, int i) const {
    if (!P.active[sc]) return;
    const BScene& s = P.scenes[sc];
    if (k >= s.nlev - 1) return;
    const BLevel F = level_of(P, s, k);
    if (j >= F.H || i >= F.W) return;
    const BLevel C = level_of(P, s, k + 1);
    const int J = j >> 1, I = i >> 1;
    int Y = J + ((j & 1) ? 1 : -1), X = I + ((i & 1) ? 1 : -1);
    Y = Y < 0 ? 0 : (Y > C.H - 1 ? C.H - 1 : Y);
    X = X < 0 ? 0 : (X > C.W - 1 ? C.W - 1 : X);
    const float* c0 = C.e + J * C.W;
    const float* c1 = C.e + Y * C.W;
    float acc = 0.0f;
    acc += 0.5625f * c0[I];
    acc += 0.1875f * c0[X];
    acc += 0.1875f * c1[I];
    acc += 0.0625f * c1[X];
    F.e[j * F.W + i] += acc;
  }
};

// r = alpha div - A p64 in float64: the next cycle's rhs (rounded to float32) and
// ||r||^2 per scene.
struct OpFineResidual {
  BPools P;
  __device__ double operator()(int sc, int j, int i) const {
    if (!P.active[sc]) return 0.0;
    const BScene& s = P.scenes[sc];
    const int H = s.H, W = s.W;
    if (j >= H || i >= W) return 0.0;
    const int64_t o = s.oc + (int64_t)j * W + i;
    const double* q = P.p64 + o;
    const double x = q[0];
    double r = s.alpha * (double)P.div[o];
    if (i > 0) r += q[-1] - x;
    if (i < W - 1) r += q[1] - x;
    if (j > 0) r += q[-W] - x;
    if (j < H - 1) r += q[W] - x;
    P.b0[o] = (float)r;
    return r * r;
  }
};

template <int TX, int TY, class F>
__global__ void __launch_bounds__(kBThreads) k_b_tiles(const BTile* __restrict__ work, int n, F f) {
  for_tiles<TX, TY>(work, n, f);
}

template <int TX, int TY, class F>
__global__ void __launch_bounds__(kBThreads) k_b_tiles_sum(const BTile* __restrict__ work, int n, double* out, F f) {
  for_tiles_sum<TX, TY>(work, n, out, f);
}

// Coarsest levels: one block per scene, e = pinv b for the scenes whose coarsest level is k.
__global__ void __launch_bounds__(kBThreads) k_b_coarse(BPools P, int k) {
  const int sc = blockIdx.x;
  if (!P.active[sc]) return;
  const BScene& s = P.scenes[sc];
  if (s.nlev - 1 != k) return;
  const BLevel L = level_of(P, s, k);
  const int n = L.H * L.W;
  const double* pinv = P.pinv + s.opinv;
  for (int row = threadIdx.x; row < n; row += blockDim.x) {
    double acc = 0.0;
    for (int q = 0; q < n; ++q) acc += pinv[(int64_t)row * n + q] * (double)L.b[q];
    L.e[row] = (float)acc;
  }
}

// Fused level kernels on 16 x 16 tiles of every scene's level k (the work list holds the
// scenes that smooth at level k): the single-grid shared-memory tile bodies with the scene's
// level arrays (row stride = row length). pre: SW sweeps from zero (or from e on a W-cycle's
// second visit), the residual and its full weighting into the coarse rhs, the smoothed
// correction into the second buffer; post: that correction plus the prolonged coarse one,
// then SW sweeps, into the level's correction. Blocks stride over the list; inactive scenes
// are skipped (whole tiles, so every barrier is block-uniform). Blocks are kTBX x kTBY
// threads, the shape the tile bodies index by.
template <int SW>
__global__ void __launch_bounds__(kTThreads) k_b_pre16(BPools P, const BTile* __restrict__ work, int n, int k,
                                                       float omega, int zero_init) {
  using S = PreShape<SW, kSX, kSY>;
  __shared__ __align__(16) float smem[4 * S::EY * S::EXh + S::XR * S::XC];
  for (int w = blockIdx.x; w < n; w += gridDim.x) {
    const BTile t = work[w];
    if (!P.active[t.scene]) continue;
    const BScene& sc = P.scenes[t.scene];
    const BLevel L = level_of(P, sc, k), C = level_of(P, sc, k + 1);
    SplitTile<float> tile =
        make_tile<float, kSX, kSY>(reinterpret_cast<unsigned char*>(smem), S::HALO, S::EXh, S::EY, L.H, L.W, t.tx, t.ty);
    float* X = smem + 4 * S::EY * S::EXh;
    const bool interior = tile.i0 >= 0 && tile.i0 + S::EX <= L.W && tile.j0 >= 0 && tile.j0 + S::EY <= L.H;
    const float* e_in = zero_init ? nullptr : L.e;
    if (interior)
      pre_body<float, SW, kSX, kSY, true>(tile, e_in, e2_of(P, sc, k), L.b, L.W, C.b, C.W, C.H, C.W, omega, X, t.tx,
                                          t.ty);
    else
      pre_body<float, SW, kSX, kSY, false>(tile, e_in, e2_of(P, sc, k), L.b, L.W, C.b, C.W, C.H, C.W, omega, X, t.tx,
                                           t.ty);
    __syncthreads();  // the next tile reuses the shared memory
  }
}

template <int SW>
__global__ void __launch_bounds__(kTThreads) k_b_post16(BPools P, const BTile* __restrict__ work, int n, int k,
                                                        float omega) {
  using S = PostShape<SW, kSX, kSY>;
  __shared__ __align__(16) float smem[4 * S::EY * S::EXh];
  for (int w = blockIdx.x; w < n; w += gridDim.x) {
    const BTile t = work[w];
    if (!P.active[t.scene]) continue;
    const BScene& sc = P.scenes[t.scene];
    const BLevel L = level_of(P, sc, k), C = level_of(P, sc, k + 1);
    SplitTile<float> tile =
        make_tile<float, kSX, kSY>(reinterpret_cast<unsigned char*>(smem), S::HALO, S::EXh, S::EY, L.H, L.W, t.tx, t.ty);
    const bool interior = tile.i0 >= 0 && tile.i0 + S::EX <= L.W && tile.j0 >= 0 && tile.j0 + S::EY <= L.H;
    if (interior)
      post_body<float, SW, kSX, kSY, true>(tile, e2_of(P, sc, k), L.e, L.b, L.W, C.e, C.W, C.H, C.W, omega);
    else
      post_body<float, SW, kSX, kSY, false>(tile, e2_of(P, sc, k), L.e, L.b, L.W, C.e, C.W, C.H, C.W, omega);
    __syncthreads();
  }
}

// Depth 0 with register tiles (the single-grid fine-level bodies, 64 x 48-cell tiles of
// every scene's fine level). pre: sweeps from zero on the rhs of the scene's cycle parity,
// residual and full weighting into level 1 (whose correction it zeroes); post: prolongation,
// sweeps, p64 += e and the next residual r - A e carried in float64 (r64) with its float32
// rounding as the next cycle's rhs, and the scene's ||r||^2 by atomic add.
using BReg = RegShape<float>;
static_assert(BReg::RPT == BReg::RPT_FINAL && BReg::NWARP == BReg::NWARP_FINAL,
              "one tile list serves the pre and the fused post kernel");

template <int SW>
__global__ void __launch_bounds__(32 * BReg::NWARP, BReg::MINB) k_b_reg_pre(BPools P, const BTile* __restrict__ work,
                                                                          int n, float omega) {
  using S = RegPre<float, SW, BReg::RPT, BReg::NWARP>;
  __shared__ RegXchg<float, BReg::NWARP> x;
  for (int w = blockIdx.x; w < n; w += gridDim.x) {
    const BTile t = work[w];
    if (!P.active[t.scene]) continue;
    const BScene& sc = P.scenes[t.scene];
    const float* bsrc = ((P.cycles[t.scene] & 1) ? P.b1 : P.b0) + sc.oc;
    const BLevel C = level_of(P, sc, 1);
    const int i0 = t.tx * S::TXO - S::HALO, j0 = t.ty * S::TYO - S::HALO;
    if (!SG_IN_BOUNDS(t.scene >= 0 && i0 + S::HALO >= 0 && i0 + S::HALO < sc.W && j0 + S::HALO < sc.H)) continue;
    const bool inside = i0 >= 0 && i0 + kRW <= sc.W && j0 >= 0 && j0 + BReg::NWARP * BReg::RPT <= sc.H;
    if (inside)
      reg_pre_body<float, SW, BReg::RPT, BReg::NWARP, false>(x, nullptr, P.e2c + sc.oc, bsrc, sc.W, sc.H, sc.W, C.b,
                                                             C.W, C.H, C.W, omega, i0, j0, C.e);
    else
      reg_pre_body<float, SW, BReg::RPT, BReg::NWARP, true>(x, nullptr, P.e2c + sc.oc, bsrc, sc.W, sc.H, sc.W, C.b,
                                                            C.W, C.H, C.W, omega, i0, j0, C.e);
    __syncthreads();  // the next tile's row exchange reuses the shared buffers
  }
}

template <int SW>
__global__ void __launch_bounds__(32 * BReg::NWARP, BReg::MINB_FINAL)
    k_b_reg_post(BPools P, const BTile* __restrict__ work, int n, float omega) {
  using S = RegPre<float, SW, BReg::RPT, BReg::NWARP>;
  __shared__ RegXchg<float, BReg::NWARP> x;
  for (int w = blockIdx.x; w < n; w += gridDim.x) {
    const BTile t = work[w];
    if (!P.active[t.scene]) continue;
    const BScene& sc = P.scenes[t.scene];
    const bool odd = P.cycles[t.scene] & 1;
    const float* bsrc = (odd ? P.b1 : P.b0) + sc.oc;
    float* bdst = (odd ? P.b0 : P.b1) + sc.oc;
    const BLevel C = level_of(P, sc, 1);
    const int i0 = t.tx * S::TXO - S::HALO, j0 = t.ty * S::TYO - S::HALO;
    if (!SG_IN_BOUNDS(t.scene >= 0 && i0 + S::HALO >= 0 && i0 + S::HALO < sc.W && j0 + S::HALO < sc.H)) continue;
    const bool inside = i0 >= 0 && i0 + kRW <= sc.W && j0 >= 0 && j0 + BReg::NWARP * BReg::RPT <= sc.H;
    double sq = 0.0;
    if (inside)
      reg_post_final_body<float, double, SW, BReg::RPT, BReg::NWARP, false>(
          x, P.e2c + sc.oc, bsrc, bdst, sc.W, sc.H, sc.W, C.e, C.W, C.H, C.W, omega, P.p64 + sc.oc, sc.W,
          P.r64 + sc.oc, i0, j0, sq);
    else
      reg_post_final_body<float, double, SW, BReg::RPT, BReg::NWARP, true>(
          x, P.e2c + sc.oc, bsrc, bdst, sc.W, sc.H, sc.W, C.e, C.W, C.H, C.W, omega, P.p64 + sc.oc, sc.W,
          P.r64 + sc.oc, i0, j0, sq);
    const double s = block_sum(sq);
    if (threadIdx.x == 0 && s != 0.0) atomicAdd(P.rn2 + t.scene, s);
    __syncthreads();
  }
}

// Depth k >= 1 on register tiles (the level kernels' bodies): pre from zero (or from the
// level's correction, on the second visit of a W-cycle) into the level's second buffer,
// zeroing level k + 1's correction; post from it plus the prolonged coarse correction into
// the level's correction. The post's halo is two cells narrower, so it has its own tiles.
template <int SW>
__global__ void __launch_bounds__(32 * BReg::NWARP, BReg::MINB) k_b_reg_pre_lev(BPools P, const BTile* __restrict__ work,
                                                                              int n, int k, float omega, int zero) {
  using S = RegPre<float, SW, BReg::RPT, BReg::NWARP>;
  __shared__ RegXchg<float, BReg::NWARP> x;
  for (int w = blockIdx.x; w < n; w += gridDim.x) {
    const BTile t = work[w];
    if (!P.active[t.scene]) continue;
    const BScene& sc = P.scenes[t.scene];
    const BLevel L = level_of(P, sc, k), C = level_of(P, sc, k + 1);
    const int i0 = t.tx * S::TXO - S::HALO, j0 = t.ty * S::TYO - S::HALO;
    if (!SG_IN_BOUNDS(t.scene >= 0 && i0 + S::HALO >= 0 && i0 + S::HALO < L.W && j0 + S::HALO < L.H)) continue;
    const bool inside = i0 >= 0 && i0 + kRW <= L.W && j0 >= 0 && j0 + BReg::NWARP * BReg::RPT <= L.H;
    if (inside)
      reg_pre_body<float, SW, BReg::RPT, BReg::NWARP, false>(x, zero ? nullptr : L.e, e2_of(P, sc, k), L.b, L.W, L.H,
                                                             L.W, C.b, C.W, C.H, C.W, omega, i0, j0, C.e);
    else
      reg_pre_body<float, SW, BReg::RPT, BReg::NWARP, true>(x, zero ? nullptr : L.e, e2_of(P, sc, k), L.b, L.W, L.H,
                                                            L.W, C.b, C.W, C.H, C.W, omega, i0, j0, C.e);
    __syncthreads();
  }
}

template <int SW>
__global__ void __launch_bounds__(32 * BReg::NWARP, BReg::MINB) k_b_reg_post_lev(BPools P, const BTile* __restrict__ work,
                                                                               int n, int k, float omega) {
  using S = RegPost<float, SW, BReg::RPT, BReg::NWARP>;
  __shared__ RegXchg<float, BReg::NWARP> x;
  for (int w = blockIdx.x; w < n; w += gridDim.x) {
    const BTile t = work[w];
    if (!P.active[t.scene]) continue;
    const BScene& sc = P.scenes[t.scene];
    const BLevel L = level_of(P, sc, k), C = level_of(P, sc, k + 1);
    const int i0 = t.tx * S::TXO - S::HALO, j0 = t.ty * S::TYO - S::HALO;
    if (!SG_IN_BOUNDS(t.scene >= 0 && i0 + S::HALO >= 0 && i0 + S::HALO < L.W && j0 + S::HALO < L.H)) continue;
    const bool inside = i0 >= 0 && i0 + kRW <= L.W && j0 >= 0 && j0 + BReg::NWARP * BReg::RPT <= L.H;
    if (inside)
      reg_post_body<float, SW, BReg::RPT, BReg::NWARP, false>(x, e2_of(P, sc, k), L.e, L.b, L.W, L.H, L.W, C.e, C.W,
                                                              C.H, C.W, omega, i0, j0);
    else
      reg_post_body<float, SW, BReg::RPT, BReg::NWARP, true>(x, e2_of(P, sc, k), L.e, L.b, L.W, L.H, L.W, C.e, C.W,
                                                             C.H, C.W, omega, i0, j0);
    __syncthreads();
  }
}

// After the rhs: ||b|| per scene, everyone starts active unless b = 0.
__global__ void k_b_start(BPools P, BCtl* ctl, cudaGraphConditionalHandle h, int use_handle) {
  int any = 0;
  for (int sc = threadIdx.x; sc < ctl->n_scenes; sc += blockDim.x) {
    const double bn2 = P.bn2[sc];
    const int act = (bn2 > 0.0 && ctl->tol < 1.0 && ctl->max_cycles > 0) ? 1 : 0;
    P.active[sc] = act;
    P.cycles[sc] = 0;
    P.relres[sc] = bn2 > 0.0 ? 1.0 : 0.0;
    P.rn2[sc] = 0.0;
    any |= act;
  }
  any = __syncthreads_or(any);
  if (threadIdx.x == 0) {
    ctl->any = any;
    if (use_handle) cudaGraphSetConditional(h, any ? 1u : 0u);
  }
}

// After a cycle: relative residual per active scene, drop the converged ones (and those at
// the cycle cap or with a non-finite residual), decide whether to run another cycle.
__global__ void k_b_after_cycle(BPools P, BCtl* ctl, cudaGraphConditionalHandle h, int use_handle) {
  int any = 0;
  for (int sc = threadIdx.x; sc < ctl->n_scenes; sc += blockDim.x) {
    if (!P.active[sc]) continue;
    const double rel = sqrt(P.rn2[sc]) / sqrt(P.bn2[sc]);
    P.rn2[sc] = 0.0;
    P.relres[sc] = rel;
    const int c = P.cycles[sc] + 1;
    P.cycles[sc] = c;
    P.total_cycles[sc] += 1;
    const bool finite = rel == rel && !isinf(rel);
    const int act = (finite && rel > ctl->tol && c < ctl->max_cycles) ? 1 : 0;
    P.active[sc] = act;
    any |= act;
  }
  any = __syncthreads_or(any);
  if (threadIdx.x == 0) {
    ctl->any = any;
    ctl->loops += 1;
    if (use_handle) cudaGraphSetConditional(h, any ? 1u : 0u);
  }
}

__global__ void k_b_clear_sums(BPools P, int n) {
  for (int sc = threadIdx.x; sc < n; sc += blockDim.x) {
    P.bn2[sc] = 0.0;
    P.rn2[sc] = 0.0;
  }
}

}  // namespace sg

// -------------------------------------------------------------- host side
struct sg_batch {
  int n = 0;
  std::vector<sg::BScene> scenes;
  int max_depth = 0;  // deepest level index over the scenes
  double tol = 1e-6;
  int max_cycles = 50;
  uint64_t seed = 0;
  float omega = 1.3f;  // red-black over-relaxation (256 scenes of 64..256 a side to 1e-6: 4.97
                       // cycles per scene and step at 1.4, 4.0 at 1.25-1.35)
  float dissipation = 0.999f;
  // layout (bytes)
  int64_t cells = 0, ufaces = 0, vfaces = 0, lev = 0, pinv_n = 0;
  std::vector<double> pinv;
  int64_t off_d[2], off_u[2], off_v[2], off_div, off_p, off_p64, off_b0, off_res, off_e, off_b, off_e2c, off_e2l,
      off_b1, off_r64, off_pinv, off_scenes,
      off_sums,
      off_ints, off_ctl, off_work, bytes = 0;
  int64_t work_cap = 0;  // tiles the work area holds
  char* ws = nullptr;
  int cur = 0;           // which of the two field buffers holds the current state
  long long step_index = 0;
  // configuration
  int tile = 0, sweeps = 2, wcycle = 0;
  // work lists of the bound configuration (device, in the work area)
  int n_cells = 0, n_faces = 0;
  int64_t lev_off[sg::kBMaxLev] = {0};
  int lev_n[sg::kBMaxLev] = {0};
  // 16 x 16 tiles of level k of the scenes that smooth there (the fused level kernels)
  int64_t lev16_off[sg::kBMaxLev] = {0};
  int lev16_n[sg::kBMaxLev] = {0};
  // depth 0 on register tiles (every scene smooths its fine level and has an even width
  // and cell count, so that the paired loads stay aligned): its tile list
  int reg0 = 0;
  int64_t reg_off = 0;
  int reg_n = 0;
  // depths 1 .. SG_BATCH_REG_TO - 1 on register tiles (every scene that smooths there has an
  // even level width and offset): their pre and post tile lists
  int regk[sg::kBMaxLev] = {0};
  int64_t regk_pre_off[sg::kBMaxLev] = {0}, regk_post_off[sg::kBMaxLev] = {0};
  int regk_pre_n[sg::kBMaxLev] = {0}, regk_post_n[sg::kBMaxLev] = {0};
  // the face tiles that can meet a scene's source disc (the sources' launch)
  int64_t src_off = 0;
  int src_n = 0;
  // graphs: one per parity of the current buffer
  cudaStream_t cs = nullptr;
  cudaGraphExec_t exec[2] = {nullptr, nullptr};
  int graph_nodes = 0, body_nodes = 0;
};

namespace sg {

static const int kTiles[][2] = {{32, 8}, {64, 4}, {16, 16}, {128, 2}};
constexpr int kNumTiles = 4;

static int64_t al256(int64_t x) { return (x + 255) & ~(int64_t)255; }

template <typename T>
static T* wsp(const sg_batch* b, int64_t off) {
  return (T*)(b->ws + off);
}

static BPools pools(const sg_batch* b) {
  BPools P;
  for (int q = 0; q < 2; ++q) {
    P.d[q] = wsp<float>(b, b->off_d[q]);
    P.u[q] = wsp<float>(b, b->off_u[q]);
    P.v[q] = wsp<float>(b, b->off_v[q]);
  }
  P.div = wsp<float>(b, b->off_div);
  P.p = wsp<float>(b, b->off_p);
  P.p64 = wsp<double>(b, b->off_p64);
  P.b0 = wsp<float>(b, b->off_b0);
  P.res = wsp<float>(b, b->off_res);
  P.e = wsp<float>(b, b->off_e);
  P.b = wsp<float>(b, b->off_b);
  P.e2c = wsp<float>(b, b->off_e2c);
  P.e2l = wsp<float>(b, b->off_e2l);
  P.b1 = wsp<float>(b, b->off_b1);
  P.r64 = wsp<double>(b, b->off_r64);
  P.pinv = wsp<double>(b, b->off_pinv);
  P.scenes = wsp<BScene>(b, b->off_scenes);
  double* sums = wsp<double>(b, b->off_sums);
  P.bn2 = sums;
  P.rn2 = sums + b->n;
  P.relres = sums + 2 * b->n;
  int* ints = wsp<int>(b, b->off_ints);
  P.active = ints;
  P.cycles = ints + b->n;
  P.total_cycles = (long long*)(b->ws + b->off_ints + al256((int64_t)8 * b->n));
  return P;
}

static BCtl* ctl_ptr(const sg_batch* b) { return wsp<BCtl>(b, b->off_ctl); }

// Tiles of every scene over rows x cols given by shape(s) (empty when rows or cols is 0).
template <class Shape>
static void add_tiles(std::vector<BTile>& out, const sg_batch* b, int TX, int TY, Shape shape) {
  for (int s = 0; s < b->n; ++s) {
    int rows = 0, cols = 0;
    shape(b->scenes[s], rows, cols);
    if (rows <= 0 || cols <= 0) continue;
    const int nty = (rows + TY - 1) / TY, ntx = (cols + TX - 1) / TX;
    for (int ty = 0; ty < nty; ++ty)
      for (int tx = 0; tx < ntx; ++tx) out.push_back(BTile{s, (short)ty, (short)tx});
  }
}

// Owned cells of a register tile for `sweeps` sweeps per side (1..3): the pre shape (also
// depth 0's fused post) or the plain post shape of the coarser depths.
template <template <typename, int, int, int> class Shape>
static void reg_tile_of(int sweeps, int& txo, int& tyo) {
  if (sweeps == 1) {
    txo = Shape<float, 1, BReg::RPT, BReg::NWARP>::TXO;
    tyo = Shape<float, 1, BReg::RPT, BReg::NWARP>::TYO;
  } else if (sweeps == 2) {
    txo = Shape<float, 2, BReg::RPT, BReg::NWARP>::TXO;
    tyo = Shape<float, 2, BReg::RPT, BReg::NWARP>::TYO;
  } else {
    txo = Shape<float, 3, BReg::RPT, BReg::NWARP>::TXO;
    tyo = Shape<float, 3, BReg::RPT, BReg::NWARP>::TYO;
  }
}
static void reg_tile(int sweeps, int& txo, int& tyo) { reg_tile_of<RegPre>(sweeps, txo, tyo); }

#ifndef SG_BATCH_REG_TO
#define SG_BATCH_REG_TO 4
#endif
// Depth k >= 1 runs on register tiles when it is below SG_BATCH_REG_TO, depth 0 does, and its
// levels allow it. (256 mixed scenes of 64..256 a side, 2 sweeps, V-cycle: 2.61 ms per step
// with depth 0 alone on register tiles, 2.31 with depth 1 too, 2.18 through depth 3, and
// no gain below: the deeper levels hold a few tiles per scene.)
static bool regk_active(const sg_batch* b, int k) {
  return k >= 1 && k < SG_BATCH_REG_TO && k < sg::kBMaxLev && b->regk[k] && b->reg0 && b->sweeps >= 1 &&
         b->sweeps <= 3;
}

// Depth 0 runs on register tiles when the batch allows it and the sweeps are 1..3.
static bool reg0_active(const sg_batch* b) { return b->reg0 && b->sweeps >= 1 && b->sweeps <= 3; }

static int build_work(sg_batch* b, cudaStream_t st) {
  const int TX = kTiles[b->tile][0], TY = kTiles[b->tile][1];
  std::vector<BTile> all;
  add_tiles(all, b, TX, TY, [](const BScene& s, int& r, int& c) { r = s.H; c = s.W; });
  b->n_cells = (int)all.size();
  add_tiles(all, b, TX, TY, [](const BScene& s, int& r, int& c) { r = s.H + 1; c = s.W + 1; });
  b->n_faces = (int)all.size() - b->n_cells;
  for (int k = 1; k <= b->max_depth; ++k) {
    b->lev_off[k] = (int64_t)all.size();
    add_tiles(all, b, TX, TY, [k](const BScene& s, int& r, int& c) {
      r = k < s.nlev ? s.lH[k] : 0;
      c = k < s.nlev ? s.lW[k] : 0;
    });
    b->lev_n[k] = (int)((int64_t)all.size() - b->lev_off[k]);
  }
  b->lev_off[0] = 0;
  b->lev_n[0] = b->n_cells;
  for (int k = 0; k < b->max_depth; ++k) {
    b->lev16_off[k] = (int64_t)all.size();
    add_tiles(all, b, kSX, kSY, [k](const BScene& s, int& r, int& c) {
      const bool smooths = k < s.nlev - 1;
      r = smooths ? (k == 0 ? s.H : s.lH[k]) : 0;
      c = smooths ? (k == 0 ? s.W : s.lW[k]) : 0;
    });
    b->lev16_n[k] = (int)((int64_t)all.size() - b->lev16_off[k]);
  }
  // source tiles: the face tiles over the disc's bounding box (a point inside the disc lies
  // within r of its centre, and the points of face (j, i) lie in [i, i + 1] x [j, j + 1])
  b->src_off = (int64_t)all.size();
  for (int sidx = 0; sidx < b->n; ++sidx) {
    const BScene& c = b->scenes[sidx];
    const double cx = c.src[0], cy = c.src[1], r = c.src[2];
    const int x0 = std::max(0, (int)std::floor(cx - r) - 2), x1 = std::min(c.W, (int)std::ceil(cx + r) + 2);
    const int y0 = std::max(0, (int)std::floor(cy - r) - 2), y1 = std::min(c.H, (int)std::ceil(cy + r) + 2);
    if (x1 < x0 || y1 < y0) continue;
    for (int ty = y0 / TY; ty <= y1 / TY; ++ty)
      for (int tx = x0 / TX; tx <= x1 / TX; ++tx) all.push_back(BTile{sidx, (short)ty, (short)tx});
  }
  b->src_n = (int)((int64_t)all.size() - b->src_off);
  b->reg_n = 0;
  if (reg0_active(b)) {
    int txo = 0, tyo = 0;
    reg_tile(b->sweeps, txo, tyo);
    b->reg_off = (int64_t)all.size();
    add_tiles(all, b, txo, tyo, [](const BScene& s, int& r, int& c) {
      r = s.nlev > 1 ? s.H : 0;
      c = s.nlev > 1 ? s.W : 0;
    });
    b->reg_n = (int)((int64_t)all.size() - b->reg_off);
  }
  for (int k = 1; k < sg::kBMaxLev; ++k) {
    b->regk_pre_n[k] = b->regk_post_n[k] = 0;
    if (!regk_active(b, k)) continue;
    auto smooth_shape = [k](const BScene& s, int& r, int& c) {
      r = k < s.nlev - 1 ? s.lH[k] : 0;
      c = k < s.nlev - 1 ? s.lW[k] : 0;
    };
    int txo = 0, tyo = 0;
    reg_tile_of<RegPre>(b->sweeps, txo, tyo);
    b->regk_pre_off[k] = (int64_t)all.size();
    add_tiles(all, b, txo, tyo, smooth_shape);
    b->regk_pre_n[k] = (int)((int64_t)all.size() - b->regk_pre_off[k]);
    reg_tile_of<RegPost>(b->sweeps, txo, tyo);
    b->regk_post_off[k] = (int64_t)all.size();
    add_tiles(all, b, txo, tyo, smooth_shape);
    b->regk_post_n[k] = (int)((int64_t)all.size() - b->regk_post_off[k]);
  }
  if ((int64_t)all.size() > b->work_cap) return fail(SG_ERR_WORKSPACE, "work list exceeds its reserved area");
  cudaError_t e = cudaMemcpyAsync(b->ws + b->off_work, all.data(), all.size() * sizeof(BTile), cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return fail(SG_ERR_CUDA, "work list upload: %s", cudaGetErrorString(e));
  return SG_OK;
}

static const BTile* work_at(const sg_batch* b, int64_t first) { return wsp<BTile>(b, b->off_work) + first; }

// Tile-list launches: one resident wave of blocks walking the list (four waves measured the
// same, a block per tile 5 % slower over the step: these tiles are short). The wave is the
// kernel's own occupancy times the SMs: with more blocks than fit at once, the rest would
// run as a second, partial wave (the tail op's 40 registers fit six blocks of 256 threads
// per SM, the scalar advection's 48 five).
template <class K>
static int resident_blocks(K kernel, int threads, size_t smem) {
  int per_sm = 0, dev = 0, sms = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem) != cudaSuccess || per_sm < 1 ||
      cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms < 1) {
    (void)cudaGetLastError();
    return 148 * (2048 / threads);
  }
  return per_sm * sms;
}

template <int TX, int TY, class F>
static int tiles_cap() {
  static const int cap = resident_blocks(k_b_tiles<TX, TY, F>, kBThreads, 0);
  return cap;
}

template <int TX, int TY, class F>
static int tiles_sum_cap() {
  static const int cap = resident_blocks(k_b_tiles_sum<TX, TY, F>, kBThreads, 0);
  return cap;
}

static unsigned grid_of(int n, int cap) { return (unsigned)std::max(1, std::min(n, cap)); }

template <int TX, int TY, class F>
static void run(const BTile* work, int n, const F& f, cudaStream_t s) {
  if (n <= 0) return;
  SG_LAUNCH(k_b_tiles<TX, TY, F><<<grid_of(n, tiles_cap<TX, TY, F>()), kBThreads, 0, s>>>(work, n, f));
}

template <int TX, int TY, class F>
static void run_sum(const BTile* work, int n, double* out, const F& f, cudaStream_t s) {
  if (n <= 0) return;
  SG_LAUNCH(k_b_tiles_sum<TX, TY, F><<<grid_of(n, tiles_sum_cap<TX, TY, F>()), kBThreads, 0, s>>>(work, n, out, f));
}

template <int SW>
static int pre16_cap() {
  static const int cap = resident_blocks(k_b_pre16<SW>, kTBX * kTBY, 0);
  return cap;
}

template <int SW>
static int post16_cap() {
  static const int cap = resident_blocks(k_b_post16<SW>, kTBX * kTBY, 0);
  return cap;
}

// The occupancy queries run once per kernel, before any stream capture.
template <int TX, int TY>
static void prime_caps() {
  tiles_cap<TX, TY, OpPlume>();
  tiles_cap<TX, TY, OpForces>();
  tiles_cap<TX, TY, OpAdvectUV>();
  tiles_cap<TX, TY, OpAdvectD>();
  tiles_cap<TX, TY, OpTail>();
  tiles_cap<TX, TY, OpRelax>();
  tiles_cap<TX, TY, OpRestrict>();
  tiles_cap<TX, TY, OpProlong>();
  tiles_cap<TX, TY, OpCorrect>();
  tiles_sum_cap<TX, TY, OpRhs>();
  tiles_sum_cap<TX, TY, OpFineResidual>();
  pre16_cap<1>(), pre16_cap<2>(), pre16_cap<3>(), pre16_cap<4>();
  post16_cap<1>(), post16_cap<2>(), post16_cap<3>(), post16_cap<4>();
}

template <int SW>
static void level_pre(const sg_batch* b, const BPools& P, int k, bool zero_init, cudaStream_t s) {
  const int n = b->lev16_n[k];
  if (n > 0)
    SG_LAUNCH(k_b_pre16<SW><<<grid_of(n, pre16_cap<SW>()), dim3(kTBX, kTBY), 0, s>>>(P, work_at(b, b->lev16_off[k]), n, k, b->omega,
                                                             zero_init ? 1 : 0));
}

template <int SW>
static void level_post(const sg_batch* b, const BPools& P, int k, cudaStream_t s) {
  const int n = b->lev16_n[k];
  if (n > 0)
    SG_LAUNCH(k_b_post16<SW><<<grid_of(n, post16_cap<SW>()), dim3(kTBX, kTBY), 0, s>>>(P, work_at(b, b->lev16_off[k]), n, k, b->omega));
}

#ifndef SG_BATCH_FUSE_FROM
#define SG_BATCH_FUSE_FROM 3
#endif
// Blocks of a register-tile launch: one per tile (the kernels keep a grid-stride loop). The
// batch step measured 2.18 ms with one resident wave of blocks walking the list, 2.11 with
// two, 2.08 with four and 2.06 with a block per tile: a block that retires early frees its
// SM slot for the next tile, where a walking block waits on its own tiles' latency.
static unsigned reg_grid(int n, int /*minb*/) { return (unsigned)std::max(1, n); }

template <int SW>
static void reg0_pre(const sg_batch* b, const BPools& P, cudaStream_t s) {
  const unsigned g = reg_grid(b->reg_n, BReg::MINB);
  SG_LAUNCH(k_b_reg_pre<SW><<<g, 32 * BReg::NWARP, 0, s>>>(P, work_at(b, b->reg_off), b->reg_n, b->omega));
}

template <int SW>
static void reg0_post(const sg_batch* b, const BPools& P, cudaStream_t s) {
  const unsigned g = reg_grid(b->reg_n, BReg::MINB_FINAL);
  SG_LAUNCH(k_b_reg_post<SW><<<g, 32 * BReg::NWARP, 0, s>>>(P, work_at(b, b->reg_off), b->reg_n, b->omega));
}

template <int SW>
static void regk_pre(const sg_batch* b, const BPools& P, int k, bool zero_init, cudaStream_t s) {
  const int n = b->regk_pre_n[k];
  if (n > 0)
    SG_LAUNCH(k_b_reg_pre_lev<SW><<<reg_grid(n, BReg::MINB), 32 * BReg::NWARP, 0, s>>>(
        P, work_at(b, b->regk_pre_off[k]), n, k, b->omega, zero_init ? 1 : 0));
}

template <int SW>
static void regk_post(const sg_batch* b, const BPools& P, int k, cudaStream_t s) {
  const int n = b->regk_post_n[k];
  if (n > 0)
    SG_LAUNCH(k_b_reg_post_lev<SW><<<reg_grid(n, BReg::MINB), 32 * BReg::NWARP, 0, s>>>(
        P, work_at(b, b->regk_post_off[k]), n, k, b->omega));
}

// Depth k of one cycle: a pre launch (sweeps, residual, restriction), the exact solve of the
// scenes whose coarsest level is k + 1, the deeper levels (twice for W), a post launch
// (prolongation, sweeps). Depth 0 and the depths below SG_BATCH_REG_TO run on register tiles
// when the batch allows it; otherwise levels k >= SG_BATCH_FUSE_FROM run the fused 16 x 16
// tile kernels, and the larger ones grid-wide half sweeps, the restriction and the
// prolongation as separate tile-list launches.
template <int TX, int TY>
static void cycle_at(const sg_batch* b, const BPools& P, int k, bool zero_init, cudaStream_t s) {
  if (regk_active(b, k)) {
    switch (b->sweeps) {
      case 1: regk_pre<1>(b, P, k, zero_init, s); break;
      case 2: regk_pre<2>(b, P, k, zero_init, s); break;
      default: regk_pre<3>(b, P, k, zero_init, s); break;
    }
    bool coarse_here = false;
    for (const BScene& sc : b->scenes) coarse_here |= sc.nlev - 1 == k + 1;
    if (coarse_here) SG_LAUNCH(k_b_coarse<<<b->n, kBThreads, 0, s>>>(P, k + 1));
    if (k + 1 < b->max_depth) {
      const int reps = b->wcycle ? 2 : 1;
      for (int q = 0; q < reps; ++q) cycle_at<TX, TY>(b, P, k + 1, q == 0, s);
    }
    switch (b->sweeps) {
      case 1: regk_post<1>(b, P, k, s); break;
      case 2: regk_post<2>(b, P, k, s); break;
      default: regk_post<3>(b, P, k, s); break;
    }
    return;
  }
  if (k == 0 && reg0_active(b)) {
    // depth 0 on register tiles; the post kernel also corrects p64 and forms the next residual
    switch (b->sweeps) {
      case 1: reg0_pre<1>(b, P, s); break;
      case 2: reg0_pre<2>(b, P, s); break;
      default: reg0_pre<3>(b, P, s); break;
    }
    bool coarse1 = false;
    for (const BScene& sc : b->scenes) coarse1 |= sc.nlev - 1 == 1;
    if (coarse1) SG_LAUNCH(k_b_coarse<<<b->n, kBThreads, 0, s>>>(P, 1));
    if (1 < b->max_depth) {
      const int reps = b->wcycle ? 2 : 1;
      for (int q = 0; q < reps; ++q) cycle_at<TX, TY>(b, P, 1, q == 0, s);
    }
    switch (b->sweeps) {
      case 1: reg0_post<1>(b, P, s); break;
      case 2: reg0_post<2>(b, P, s); break;
      default: reg0_post<3>(b, P, s); break;
    }
    return;
  }
  const bool fused = k >= SG_BATCH_FUSE_FROM;
  const BTile* lw = work_at(b, b->lev_off[k]);
  const int ln = b->lev_n[k];
  if (fused) {
    switch (b->sweeps) {
      case 1: level_pre<1>(b, P, k, zero_init, s); break;
      case 2: level_pre<2>(b, P, k, zero_init, s); break;
      case 3: level_pre<3>(b, P, k, zero_init, s); break;
      default: level_pre<4>(b, P, k, zero_init, s); break;
    }
  } else {
    for (int sw = 0; sw < b->sweeps; ++sw)
      for (int c = 0; c < 2; ++c) run<TX, TY>(lw, ln, OpRelax{P, k, c, b->omega}, s);
    run<TX, TY>(work_at(b, b->lev_off[k + 1]), b->lev_n[k + 1], OpRestrict{P, k}, s);
  }
  bool coarse_here = false;
  for (const BScene& sc : b->scenes) coarse_here |= sc.nlev - 1 == k + 1;
  if (coarse_here) SG_LAUNCH(k_b_coarse<<<b->n, kBThreads, 0, s>>>(P, k + 1));
  if (k + 1 < b->max_depth) {
    const int reps = b->wcycle ? 2 : 1;
    for (int q = 0; q < reps; ++q) cycle_at<TX, TY>(b, P, k + 1, q == 0, s);
  }
  if (fused) {
    switch (b->sweeps) {
      case 1: level_post<1>(b, P, k, s); break;
      case 2: level_post<2>(b, P, k, s); break;
      case 3: level_post<3>(b, P, k, s); break;
      default: level_post<4>(b, P, k, s); break;
    }
  } else {
    run<TX, TY>(lw, ln, OpProlong{P, k}, s);
    for (int sw = 0; sw < b->sweeps; ++sw)
      for (int c = 0; c < 2; ++c) run<TX, TY>(lw, ln, OpRelax{P, k, c, b->omega}, s);
  }
}

// One step with the current state in buffer `cur`: everything up to the solve.
template <int TX, int TY>
static void step_head(const sg_batch* b, const BPools& P, int cur, long long step, cudaStream_t s) {
  const BTile* cw = work_at(b, 0);
  const BTile* fw = work_at(b, b->n_cells);
  run<TX, TY>(work_at(b, b->src_off), b->src_n, OpPlume{P, cur, b->seed, step < 0 ? 0 : step}, s);
  run<TX, TY>(fw, b->n_faces, OpForces{P, cur}, s);
  run<TX, TY>(fw, b->n_faces, OpAdvectUV{P}, s);
  run<TX, TY>(cw, b->n_cells, OpAdvectD{P, cur, b->dissipation}, s);
  SG_LAUNCH(k_b_clear_sums<<<1, 1024, 0, s>>>(P, b->n));
  run_sum<TX, TY>(cw, b->n_cells, P.bn2, OpRhs{P, reg0_active(b) ? 0 : 1}, s);
}

template <int TX, int TY>
static void solve_body(const sg_batch* b, const BPools& P, cudaGraphConditionalHandle h, int use_handle,
                       cudaStream_t s) {
  if (b->max_depth == 0) {
    SG_LAUNCH(k_b_coarse<<<b->n, kBThreads, 0, s>>>(P, 0));
  } else {
    cycle_at<TX, TY>(b, P, 0, true, s);
  }
  if (!reg0_active(b)) {  // (the register-tiled depth 0 did both in its post kernel)
    run<TX, TY>(work_at(b, 0), b->n_cells, OpCorrect{P}, s);
    run_sum<TX, TY>(work_at(b, 0), b->n_cells, P.rn2, OpFineResidual{P}, s);
  }
  SG_LAUNCH(k_b_after_cycle<<<1, 1024, 0, s>>>(P, ctl_ptr(b), h, use_handle));
}

template <int TX, int TY>
static void step_tail(const sg_batch* b, const BPools& P, cudaStream_t s) {
  run<TX, TY>(work_at(b, 0), b->n_cells, OpTail{P}, s);
}

#define SG_BTRY(x, what)                                                                  \
  do {                                                                                    \
    cudaError_t _e = (x);                                                                 \
    if (_e != cudaSuccess) return fail(SG_ERR_CUDA, "%s: %s", what, cudaGetErrorString(_e)); \
  } while (0)

// Graph of one step starting from buffer `cur`: head, WHILE(any scene active) cycle, tail.
template <int TX, int TY>
static int build_step_graph(sg_batch* b, int cur, cudaGraphExec_t* out) {
  prime_caps<TX, TY>();
  BPools P = pools(b);
  cudaStream_t cs = b->cs;
  cudaGraph_t g = nullptr;
  SG_BTRY(cudaGraphCreate(&g, 0), "cudaGraphCreate");
  cudaGraphConditionalHandle h;
  SG_BTRY(cudaGraphConditionalHandleCreate(&h, g, 0, 0), "conditional handle");
  SG_BTRY(cudaStreamBeginCaptureToGraph(cs, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal), "capture");
  unsigned long long c0 = launch_count();
  // the step index travels in device memory (graph launches reuse the same parameters)
  step_head<TX, TY>(b, P, cur, -1, cs);
  SG_LAUNCH(k_b_start<<<1, 1024, 0, cs>>>(P, ctl_ptr(b), h, 1));
  cudaStreamCaptureStatus cst;
  cudaGraph_t cg = nullptr;
  const cudaGraphNode_t* deps = nullptr;
  size_t ndeps = 0;
  SG_BTRY(cudaStreamGetCaptureInfo(cs, &cst, nullptr, &cg, &deps, &ndeps), "capture info");
  alignas(cudaGraphNodeParams) unsigned char buf[sizeof(cudaGraphNodeParams)];
  std::memset(buf, 0, sizeof(buf));
  cudaGraphNodeParams& cp = *reinterpret_cast<cudaGraphNodeParams*>(buf);
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t cnode;
  SG_BTRY(cudaGraphAddNode(&cnode, cg, deps, ndeps, &cp), "conditional node");
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  SG_BTRY(cudaStreamUpdateCaptureDependencies(cs, &cnode, 1, cudaStreamSetCaptureDependencies), "deps");
  step_tail<TX, TY>(b, P, cs);
  unsigned long long c1 = launch_count();
  SG_BTRY(cudaStreamEndCapture(cs, &g), "end capture");
  SG_BTRY(cudaStreamBeginCaptureToGraph(cs, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal),
          "body capture");
  solve_body<TX, TY>(b, P, h, 1, cs);
  unsigned long long c2 = launch_count();
  SG_BTRY(cudaStreamEndCapture(cs, &body), "end body capture");
  cudaError_t e = cudaGraphInstantiate(out, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return fail(SG_ERR_CUDA, "cudaGraphInstantiate: %s", cudaGetErrorString(e));
  b->graph_nodes = (int)(c1 - c0);
  b->body_nodes = (int)(c2 - c1);
  return SG_OK;
}

static int build_graphs(sg_batch* b) {
  for (int q = 0; q < 2; ++q)
    if (b->exec[q]) {
      cudaGraphExecDestroy(b->exec[q]);
      b->exec[q] = nullptr;
    }
  if (!b->cs) SG_BTRY(cudaStreamCreateWithFlags(&b->cs, cudaStreamNonBlocking), "stream");
  int rc = build_work(b, b->cs);
  if (rc != SG_OK) return rc;
  SG_BTRY(cudaStreamSynchronize(b->cs), "work list upload");
  for (int q = 0; q < 2; ++q) {
    switch (b->tile) {
      case 0: rc = build_step_graph<32, 8>(b, q, &b->exec[q]); break;
      case 1: rc = build_step_graph<64, 4>(b, q, &b->exec[q]); break;
      case 2: rc = build_step_graph<16, 16>(b, q, &b->exec[q]); break;
      default: rc = build_step_graph<128, 2>(b, q, &b->exec[q]); break;
    }
    if (rc != SG_OK) return rc;
  }
  return SG_OK;
}

// The step index the plume noise hashes is read from the control block.
static int launch_steps(sg_batch* b, int n, cudaStream_t s) {
  for (int k = 0; k < n; ++k) {
    SG_BTRY(cudaGraphLaunch(b->exec[b->cur], s), "cudaGraphLaunch");
    b->cur = 1 - b->cur;
    b->step_index += 1;
  }
  return check_launch("sg_batch_step");
}

}  // namespace sg

using namespace sg;

extern "C" {

int sg_batch_create(sg_batch** out, int n_scenes, const int* H, const int* W, const double* params, double tol,
                    int max_cycles, uint64_t seed) {
  SG_REQUIRE(out, "null batch pointer");
  *out = nullptr;
  SG_REQUIRE(n_scenes >= 1 && n_scenes <= (1 << 20) && H && W && params, "bad scene table");
  SG_REQUIRE(tol > 0.0 && tol < 1.0 && max_cycles >= 1 && max_cycles <= 1000, "bad tolerance / cycle cap");
  sg_batch* b = new sg_batch();
  b->n = n_scenes;
  b->tol = tol;
  b->max_cycles = max_cycles;
  b->seed = seed;
  b->scenes.resize(n_scenes);
  std::vector<std::pair<int, int>> shapes;  // distinct coarsest shapes
  std::vector<int64_t> shape_off;
  for (int s = 0; s < n_scenes; ++s) {
    BScene& c = b->scenes[s];
    std::memset(&c, 0, sizeof(c));
    if (H[s] < 2 || W[s] < 2 || H[s] > 8192 || W[s] > 8192 || (int64_t)H[s] / 32 > 32767) {
      delete b;
      return fail(SG_ERR_ARG, "scene %d: grid must be 2..8192 cells a side", s);
    }
    const double* q = params + 10 * s;  // h, dt, rho, gravity, buoyancy, cx, cy, r, density, v_in
    if (!(q[0] > 0.0 && q[1] > 0.0 && q[2] > 0.0)) {
      delete b;
      return fail(SG_ERR_ARG, "scene %d: cell size, dt and density must be positive", s);
    }
    c.H = H[s];
    c.W = W[s];
    c.inv = 1.0 / q[0];
    c.dt = q[1];
    c.alpha = -(q[0] * q[0]) * q[2] / q[1];
    c.scale = q[1] / (q[2] * q[0]);
    c.gravity = q[3];
    c.dcoef = q[4];
    c.src[0] = q[5];
    c.src[1] = q[6];
    c.src[2] = q[7];
    c.src[3] = q[8];
    c.src[4] = q[9];
    c.src[5] = 0.0;
    // hierarchy: halve (rounding up) until no side exceeds 8
    int h = c.H, w = c.W, k = 0;
    c.lH[0] = h;
    c.lW[0] = w;
    while (std::max(h, w) > 8) {
      if (k + 1 >= kBMaxLev) {
        delete b;
        return fail(SG_ERR_CAPACITY, "scene %d needs more than %d levels", s, kBMaxLev);
      }
      h = (h + 1) / 2;
      w = (w + 1) / 2;
      ++k;
      c.lH[k] = h;
      c.lW[k] = w;
    }
    c.nlev = k + 1;
    b->max_depth = std::max(b->max_depth, k);
    c.oc = b->cells;
    c.ou = b->ufaces;
    c.ov = b->vfaces;
    b->cells += (int64_t)c.H * c.W;
    b->ufaces += (int64_t)c.H * (c.W + 1);
    b->vfaces += (int64_t)(c.H + 1) * c.W;
    for (int q2 = 1; q2 < c.nlev; ++q2) {
      c.olev[q2] = b->lev;
      b->lev += (int64_t)c.lH[q2] * c.lW[q2];
    }
    auto key = std::make_pair(h, w);
    auto it = std::find(shapes.begin(), shapes.end(), key);
    if (it == shapes.end()) {
      std::vector<double> pv;
      if (!open_box_pinv(h, w, pv)) {
        delete b;
        return fail(SG_ERR_ARG, "coarsest %d x %d could not be factorised", h, w);
      }
      shapes.push_back(key);
      shape_off.push_back((int64_t)b->pinv.size());
      b->pinv.insert(b->pinv.end(), pv.begin(), pv.end());
      it = shapes.end() - 1;
    }
    c.opinv = shape_off[it - shapes.begin()];
  }
  // depth 0 on register tiles: every scene smooths its fine level, and every width and cell
  // count is even (the tiles' paired loads and stores need even element offsets)
  b->reg0 = 1;
  for (const BScene& c : b->scenes)
    if (c.nlev < 2 || (c.W & 1) || ((int64_t)c.H * c.W) & 1) b->reg0 = 0;
  for (int k = 1; k < kBMaxLev; ++k) {
    b->regk[k] = k <= b->max_depth ? 1 : 0;
    for (const BScene& c : b->scenes)
      if (k < c.nlev - 1 && ((c.lW[k] & 1) || (c.olev[k] & 1))) b->regk[k] = 0;
  }
  // work area: every scene's cell, face and level tiles under its most fragmenting shape
  b->work_cap = 0;
  for (const BScene& c : b->scenes) {
    int64_t best = 0;
    for (int t = 0; t < kNumTiles; ++t) {
      const int TX = kTiles[t][0], TY = kTiles[t][1];
      int64_t n = (int64_t)((c.H + TY - 1) / TY) * ((c.W + TX - 1) / TX) +
                  (int64_t)((c.H + TY) / TY) * ((c.W + TX) / TX);
      for (int k = 1; k < c.nlev; ++k) n += (int64_t)((c.lH[k] + TY - 1) / TY) * ((c.lW[k] + TX - 1) / TX);
      best = std::max(best, n);
    }
    b->work_cap += best;
    for (int k = 0; k + 1 < c.nlev; ++k) {  // the fused level kernels' 16 x 16 tiles
      const int h = k == 0 ? c.H : c.lH[k], w = k == 0 ? c.W : c.lW[k];
      b->work_cap += (int64_t)((h + kSY - 1) / kSY) * ((w + kSX - 1) / kSX);
    }
    {  // source tiles: at most every face tile of the scene, under the smallest tile shape
      int64_t most = 0;
      for (int t = 0; t < kNumTiles; ++t)
        most = std::max(most, (int64_t)((c.H + kTiles[t][1]) / kTiles[t][1] + 1) * ((c.W + kTiles[t][0]) / kTiles[t][0] + 1));
      b->work_cap += most;
    }
    {  // register tiles at their smallest (3 sweeps; the pre shape bounds the post's too)
      int txo = 0, tyo = 0;
      reg_tile(3, txo, tyo);
      b->work_cap += (int64_t)((c.H + tyo - 1) / tyo) * ((c.W + txo - 1) / txo);
      for (int k = 1; k + 1 < c.nlev && k < SG_BATCH_REG_TO; ++k)
        b->work_cap += 2 * (int64_t)((c.lH[k] + tyo - 1) / tyo) * ((c.lW[k] + txo - 1) / txo);
    }
  }
  int64_t off = 0;
  auto take = [&](int64_t bytes) {
    int64_t o = off;
    off = al256(off + bytes);
    return o;
  };
  for (int q = 0; q < 2; ++q) {
    b->off_d[q] = take(4 * b->cells);
    b->off_u[q] = take(4 * b->ufaces);
    b->off_v[q] = take(4 * b->vfaces);
  }
  b->off_div = take(4 * b->cells);
  b->off_p = take(4 * b->cells);
  b->off_p64 = take(8 * b->cells);
  b->off_b0 = take(4 * b->cells);
  b->off_res = take(4 * b->cells);
  b->off_e = take(4 * std::max<int64_t>(b->lev, 1));
  b->off_b = take(4 * std::max<int64_t>(b->lev, 1));
  b->off_e2c = take(4 * b->cells);
  b->off_e2l = take(4 * std::max<int64_t>(b->lev, 1));
  b->off_b1 = take(4 * b->cells);
  b->off_r64 = take(8 * b->cells);
  b->off_pinv = take(8 * (int64_t)b->pinv.size());
  b->off_scenes = take((int64_t)sizeof(BScene) * n_scenes);
  b->off_sums = take(8 * 3 * (int64_t)n_scenes);
  b->off_ints = take(al256((int64_t)8 * n_scenes) + 8 * (int64_t)n_scenes);
  b->off_ctl = take(sizeof(BCtl));
  b->off_work = take((int64_t)sizeof(BTile) * b->work_cap);
  b->bytes = off;
  *out = b;
  return SG_OK;
}

void sg_batch_destroy(sg_batch* b) {
  if (!b) return;
  for (int q = 0; q < 2; ++q)
    if (b->exec[q]) cudaGraphExecDestroy(b->exec[q]);
  if (b->cs) cudaStreamDestroy(b->cs);
  delete b;
}

int64_t sg_batch_workspace_bytes(const sg_batch* b) { return b ? b->bytes : -1; }

int sg_batch_layout(const sg_batch* b, int scene, int64_t* off_density, int64_t* off_u, int64_t* off_v,
                    int64_t* off_pressure) {
  SG_REQUIRE(b && scene >= 0 && scene < b->n, "bad batch / scene");
  const BScene& c = b->scenes[scene];
  const int q = b->cur;
  if (off_density) *off_density = b->off_d[q] + 4 * c.oc;
  if (off_u) *off_u = b->off_u[kVel] + 4 * c.ou;
  if (off_v) *off_v = b->off_v[kVel] + 4 * c.ov;
  if (off_pressure) *off_pressure = b->off_p + 4 * c.oc;
  return SG_OK;
}

int sg_batch_bind(sg_batch* b, void* workspace, int64_t bytes, void* stream) {
  SG_REQUIRE(b && workspace, "null batch / workspace");
  SG_REQUIRE(bytes >= b->bytes, "workspace of %lld bytes below the %lld needed", (long long)bytes,
             (long long)b->bytes);
  SG_REQUIRE(((uintptr_t)workspace & 255) == 0, "workspace must be 256-byte aligned");
  cudaStream_t s = as_stream(stream);
  b->ws = (char*)workspace;
  b->cur = 0;
  b->step_index = 0;
  SG_BTRY(cudaMemsetAsync(b->ws, 0, b->off_pinv, s), "zero fields");
  SG_BTRY(cudaMemcpyAsync(b->ws + b->off_pinv, b->pinv.data(), 8 * b->pinv.size(), cudaMemcpyHostToDevice, s),
          "pinv upload");
  SG_BTRY(cudaMemcpyAsync(b->ws + b->off_scenes, b->scenes.data(), sizeof(BScene) * b->n, cudaMemcpyHostToDevice, s),
          "scene upload");
  SG_BTRY(cudaMemsetAsync(b->ws + b->off_sums, 0, b->off_work - b->off_sums, s), "zero state");
  BCtl ctl;
  std::memset(&ctl, 0, sizeof(ctl));
  ctl.tol = b->tol;
  ctl.max_cycles = b->max_cycles;
  ctl.n_scenes = b->n;
  SG_BTRY(cudaMemcpyAsync(b->ws + b->off_ctl, &ctl, sizeof(ctl), cudaMemcpyHostToDevice, s), "control upload");
  SG_BTRY(cudaStreamSynchronize(s), "bind");
  return build_graphs(b);
}

int sg_batch_configure(sg_batch* b, int tile, int sweeps, int wcycle) {
  SG_REQUIRE(b && b->ws, "batch not bound");
  SG_REQUIRE(tile >= 0 && tile < kNumTiles, "tile must be 0..%d", kNumTiles - 1);
  SG_REQUIRE(sweeps >= 1 && sweeps <= 4, "sweeps must be 1..4");
  SG_REQUIRE(wcycle == 0 || wcycle == 1, "cycle must be 0 (V) or 1 (W)");
  b->tile = tile;
  b->sweeps = sweeps;
  b->wcycle = wcycle;
  return build_graphs(b);
}

int sg_batch_tile_shape(int tile, int* tx, int* ty) {
  SG_REQUIRE(tile >= 0 && tile < kNumTiles && tx && ty, "bad tile index");
  *tx = kTiles[tile][0];
  *ty = kTiles[tile][1];
  return SG_OK;
}

int sg_batch_step(sg_batch* b, int n_steps, void* stream) {
  SG_REQUIRE(b && b->ws && b->exec[0], "batch not bound");
  SG_REQUIRE(n_steps >= 0, "n_steps must be >= 0");
  return launch_steps(b, n_steps, as_stream(stream));
}

int sg_batch_current(const sg_batch* b) { return b ? b->cur : -1; }

// Cycle-loop iterations (one per cycle of all scenes together) run since bind; synchronises.
int sg_batch_loops(sg_batch* b, long long* loops, void* stream) {
  SG_REQUIRE(b && b->ws && loops, "batch not bound");
  cudaStream_t s = as_stream(stream);
  SG_BTRY(cudaMemcpyAsync(loops, &ctl_ptr(b)->loops, sizeof(long long), cudaMemcpyDeviceToHost, s), "loops");
  SG_BTRY(cudaStreamSynchronize(s), "loops");
  return SG_OK;
}

int sg_batch_graph_nodes(const sg_batch* b, int* step_nodes, int* cycle_nodes) {
  SG_REQUIRE(b && step_nodes && cycle_nodes, "null pointer");
  *step_nodes = b->graph_nodes;
  *cycle_nodes = b->body_nodes;
  return SG_OK;
}

// Per-scene solve outcome of the last step (host arrays of n entries, any may be NULL);
// synchronises the stream.
int sg_batch_stats(sg_batch* b, int* cycles, double* relres, long long* total_cycles, void* stream) {
  SG_REQUIRE(b && b->ws, "batch not bound");
  cudaStream_t s = as_stream(stream);
  BPools P = pools(b);
  if (cycles) SG_BTRY(cudaMemcpyAsync(cycles, P.cycles, 4 * b->n, cudaMemcpyDeviceToHost, s), "stats");
  if (relres) SG_BTRY(cudaMemcpyAsync(relres, P.relres, 8 * b->n, cudaMemcpyDeviceToHost, s), "stats");
  if (total_cycles) SG_BTRY(cudaMemcpyAsync(total_cycles, P.total_cycles, 8 * b->n, cudaMemcpyDeviceToHost, s), "stats");
  SG_BTRY(cudaStreamSynchronize(s), "stats");
  return SG_OK;
}

int64_t sg_batch_snapshot_bytes(const sg_batch* b) { return b ? b->off_pinv : -1; }

// Autotuner: time `steps` steps of every (tile, sweeps, cycle) candidate from the current
// state (restored from `scratch`, sg_batch_snapshot_bytes bytes, after each), keep the
// fastest whose scenes all converged; returns the choice and its time per step. The state
// is left as it was.
int sg_batch_autotune(sg_batch* b, int steps, void* scratch, int64_t scratch_bytes, void* stream, int* tile,
                      int* sweeps, int* wcycle, double* ms_per_step) {
  SG_REQUIRE(b && b->ws, "batch not bound");
  SG_REQUIRE(steps >= 1 && steps <= 100, "steps must be 1..100");
  SG_REQUIRE(scratch && scratch_bytes >= b->off_pinv, "scratch below sg_batch_snapshot_bytes()");
  cudaStream_t s = as_stream(stream);
  // snapshot of everything the steps change (the field pools)
  const int64_t span = b->off_pinv;
  char* snap = (char*)scratch;
  SG_BTRY(cudaMemcpyAsync(snap, b->ws, span, cudaMemcpyDeviceToDevice, s), "snapshot");
  const int cur0 = b->cur;
  const long long step0 = b->step_index;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  double best = 1e300;
  int bt = b->tile, bs = b->sweeps, bw = b->wcycle;
  int rc = SG_OK;
  std::vector<int> cyc(b->n);
  for (int t = 0; t < kNumTiles && rc == SG_OK; ++t)
    for (int sw = 1; sw <= 3 && rc == SG_OK; ++sw)
      for (int w = 0; w <= 1 && rc == SG_OK; ++w) {
        b->tile = t;
        b->sweeps = sw;
        b->wcycle = w;
        rc = build_graphs(b);
        if (rc != SG_OK) break;
        // warm-up step, then the timed ones, each from the snapshot
        for (int pass = 0; pass < 2 && rc == SG_OK; ++pass) {
          if (cudaMemcpyAsync(b->ws, snap, span, cudaMemcpyDeviceToDevice, s) != cudaSuccess) rc = SG_ERR_CUDA;
          b->cur = cur0;
          b->step_index = step0;
          cudaEventRecord(e0, s);
          if (rc == SG_OK) rc = launch_steps(b, pass == 0 ? 1 : steps, s);
          cudaEventRecord(e1, s);
        }
        if (rc != SG_OK) break;
        cudaEventSynchronize(e1);
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        rc = sg_batch_stats(b, cyc.data(), nullptr, nullptr, stream);
        bool ok = true;
        for (int c : cyc) ok &= c < b->max_cycles;
        const double per = ms / steps;
        if (ok && per < best) {
          best = per;
          bt = t;
          bs = sw;
          bw = w;
        }
      }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaMemcpyAsync(b->ws, snap, span, cudaMemcpyDeviceToDevice, s);
  b->cur = cur0;
  b->step_index = step0;
  if (rc != SG_OK) return rc;
  b->tile = bt;
  b->sweeps = bs;
  b->wcycle = bw;
  rc = build_graphs(b);
  if (tile) *tile = bt;
  if (sweeps) *sweeps = bs;
  if (wcycle) *wcycle = bw;
  if (ms_per_step) *ms_per_step = best;
  return rc;
}

}  // extern "C"

SG_BOUNDS_ACCESSOR(batch)
