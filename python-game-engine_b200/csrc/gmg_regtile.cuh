// Register-tiled level kernels of the convergent multigrid for large open-box levels
// (included inside namespace sg by gmg.cu, and by batch.cu with SG_REGTILE_BODIES_ONLY for
// the device bodies alone; uses w1 and rcp_open of gmg_weights.cuh).
//
// Same two launches per level and cycle as the shared-memory tiles (pre: sweeps + residual
// + full weighting; post: prolongation + sweeps), but the cells stay in registers:
//   - a block is NWARP warps stacked vertically over a 64-column tile; lane l owns columns
//     i0 + 2l, i0 + 2l + 1 and warp w owns rows j0 + w RPT .. j0 + w RPT + RPT - 1;
//   - horizontal neighbours come from the adjacent lane by warp shuffles, vertical ones from
//     the thread's own registers, except the first and last row of a warp, which are
//     exchanged through shared memory once per half sweep (one barrier, double-buffered);
//   - the tile origin (i0, j0) is even, so the colour of a register cell, (r + q) & 1, is
//     known at compile time and every half sweep is straight-line code.
// The tile carries a halo (pre: 2 SW + 2 cells, post: 2 SW) that absorbs the wrong values
// grown from its edge, one cell per half sweep, so every cell a block writes holds exactly
// what grid-wide half sweeps give. Blocks read e from one buffer and write another (pre:
// E0 or nothing -> E1, post: E1 -> E0), so no block reads cells another one is writing.
// Tiles whose cells all lie inside the grid take a path without bounds checks; on the
// others, cells outside the grid hold 0 and are never updated, so the relaxation sum is
// unchanged and only the neighbour count (and the residual's terms) need the bounds.
#pragma once

constexpr int kRW = 64;  // tile columns: 32 lanes x 2

// The first cycle of a solve from a zero guess, for the fused fine-level post kernel: p is 0
// on entry (not read), and when div is set the carried float64 residual r64 starts as
// alpha div (- the fluid mean with sub_mean), formed here from the divergence instead of being
// written by the prologue and read back. div: float32 (f64 = 0) or float64 values, row stride
// ldd. active = 0: an ordinary cycle. alpha and mean are filled in on the device from the
// solve state by the kernel that takes the struct.
struct FirstCycle {
  const void* div;
  int64_t ldd;
  int f64;
  int sub_mean;
  int active;
  double alpha, mean;
};
__device__ __forceinline__ double first_cycle_rhs(const FirstCycle& fc, int64_t o) {
  const double d = fc.f64 ? ((const double*)fc.div)[o] : (double)((const float*)fc.div)[o];
  double x = fc.alpha * d;
  if (fc.sub_mean) x -= fc.mean;
  return x;
}

template <typename T>
struct Pair;
template <>
struct Pair<float> {
  using V = float2;
};
template <>
struct Pair<double> {
  using V = double2;
};

template <typename T>
__device__ __forceinline__ T shfl_up1(T v) {
  return __shfl_up_sync(0xffffffffu, v, 1);
}
template <typename T>
__device__ __forceinline__ T shfl_down1(T v) {
  return __shfl_down_sync(0xffffffffu, v, 1);
}

// Shared-memory exchange of the first and last row of each warp (double-buffered).
template <typename T, int NWARP>
struct RegXchg {
  typename Pair<T>::V top[2][NWARP][32];
  typename Pair<T>::V bot[2][NWARP][32];
  T xtop[NWARP][32];
  T xbot[NWARP][32];
};

// Synchronisation of the row exchange: the block-wide barrier by default. With
// SG_REG_PAIR_SYNC=1 each pair of adjacent warps shares one named barrier instead (id w for
// warps w - 1 and w, 64 threads), so a warp waits for its two neighbours only. A warp takes
// its upper barrier before its lower one: warp 0 has no upper one, so the chain always
// completes; double buffering stays safe, since a warp rewrites buffer buf only after the
// next exchange's barriers with both neighbours, which they reach after reading buf.
// Measured at 2048^2 (mixed, ncu launch list): the pair barriers made the register-tile
// kernels slower (fine post 42.9 -> 44.1 us, pre 12.8 -> 13.4 us, 1024^2 post 9.2 -> 10.3 us).
#ifndef SG_REG_PAIR_SYNC
#define SG_REG_PAIR_SYNC 0
#endif
template <int NWARP>
__device__ __forceinline__ void sync_neighbour_warps(int w) {
#if SG_REG_PAIR_SYNC
  static_assert(NWARP <= 16, "one named barrier per warp edge (ids 1 .. NWARP - 1)");
  if (w > 0) asm volatile("bar.sync %0, 64;" ::"r"(w) : "memory");
  if (w < NWARP - 1) asm volatile("bar.sync %0, 64;" ::"r"(w + 1) : "memory");
#else
  __syncthreads();
#endif
}

// Publish the warp's edge rows into buffer buf, wait, and fetch the neighbouring warps'
// edges: above = row w RPT - 1 (last row of warp w - 1), below = row (w + 1) RPT (first row
// of warp w + 1). The outermost warps get their own rows back (halo cells, never used).
template <typename T, int RPT, int NWARP>
__device__ __forceinline__ void exchange_rows(RegXchg<T, NWARP>& x, int buf, const T (&e)[RPT][2], int w, int lane,
                                              T (&above)[2], T (&below)[2]) {
  using V = typename Pair<T>::V;
  V t, bo;
  t.x = e[0][0];
  t.y = e[0][1];
  bo.x = e[RPT - 1][0];
  bo.y = e[RPT - 1][1];
  x.top[buf][w][lane] = t;
  x.bot[buf][w][lane] = bo;
  sync_neighbour_warps<NWARP>(w);
  const V a = x.bot[buf][w > 0 ? w - 1 : w][lane];
  const V b = x.top[buf][w < NWARP - 1 ? w + 1 : w][lane];
  above[0] = a.x;
  above[1] = a.y;
  below[0] = b.x;
  below[1] = b.y;
}

// One half sweep of colour COL over the thread's cells. Row r, column q has colour
// (r + q) & 1. BOUNDED: tile touches the grid edge; (j, i) of the thread's first cell.
template <typename T, int RPT, int COL, bool BOUNDED>
__device__ __forceinline__ void reg_half_sweep(T (&e)[RPT][2], const T (&b)[RPT][2], const T (&above)[2],
                                               const T (&below)[2], T omega, int j, int i, int H, int W) {
#pragma unroll
  for (int r = 0; r < RPT; ++r) {
    const int q = (COL + r) & 1;
    // the neighbour in the other lane: q = 0 needs column 2l - 1 (lane l - 1's column 1),
    // q = 1 needs column 2l + 2 (lane l + 1's column 0)
    const T far = q == 0 ? shfl_up1(e[r][1]) : shfl_down1(e[r][0]);
    const T left = q == 0 ? far : e[r][0];
    const T right = q == 0 ? e[r][1] : far;
    const T up = r > 0 ? e[r > 0 ? r - 1 : 0][q] : above[q];
    const T down = r < RPT - 1 ? e[r < RPT - 1 ? r + 1 : 0][q] : below[q];
    const T acc = b[r][q] + left + right + up + down;
    const T x = e[r][q];
    if (!BOUNDED) {
      e[r][q] = x + omega * (acc * (T)0.25 - x);
    } else {
      const int jj = j + r, ii = i + q;
      if (jj >= 0 && jj < H && ii >= 0 && ii < W) {
        const int n = (ii > 0) + (ii < W - 1) + (jj > 0) + (jj < H - 1);
        if (n > 0) e[r][q] = x + omega * (acc * rcp_open<T>(n) - x);
      }
    }
  }
}

// The first half sweep (colour 0) from e = 0: every neighbour is 0, so the update is
// omega * (b * 1/n) (the general formula with x = 0 and a zero neighbour sum: the same
// value, up to the sign of a zero) and needs no row exchange.
template <typename T, int RPT, bool BOUNDED>
__device__ __forceinline__ void reg_first_half_sweep_from_zero(T (&e)[RPT][2], const T (&b)[RPT][2], T omega, int j,
                                                               int i, int H, int W) {
#pragma unroll
  for (int r = 0; r < RPT; ++r) {
    const int q = r & 1;
    if (!BOUNDED) {
      e[r][q] = omega * (b[r][q] * (T)0.25);
    } else {
      const int jj = j + r, ii = i + q;
      if (jj >= 0 && jj < H && ii >= 0 && ii < W) {
        const int n = (ii > 0) + (ii < W - 1) + (jj > 0) + (jj < H - 1);
        if (n > 0) e[r][q] = omega * (b[r][q] * rcp_open<T>(n));
      }
    }
  }
}

template <typename T, int RPT, int NWARP, int NHS, int HS, bool BOUNDED>
__device__ __forceinline__ void reg_sweeps(RegXchg<T, NWARP>& x, T (&e)[RPT][2], const T (&b)[RPT][2], T omega,
                                           int w, int lane, int j, int i, int H, int W) {
  if constexpr (HS < NHS) {
    T above[2], below[2];
    exchange_rows<T, RPT, NWARP>(x, HS & 1, e, w, lane, above, below);
    reg_half_sweep<T, RPT, HS & 1, BOUNDED>(e, b, above, below, omega, j, i, H, W);
    reg_sweeps<T, RPT, NWARP, NHS, HS + 1, BOUNDED>(x, e, b, omega, w, lane, j, i, H, W);
  }
}

// Load RPT x 2 cells at (j, i) (i even) from a level array; cells outside the grid get 0.
template <typename T, int RPT, bool BOUNDED>
__device__ __forceinline__ void reg_load(T (&v)[RPT][2], const T* __restrict__ a, int64_t ld, int j, int i, int H,
                                         int W) {
  using V = typename Pair<T>::V;
#pragma unroll
  for (int r = 0; r < RPT; ++r) {
    const int jj = j + r;
    if (!BOUNDED) {
      if (SG_IN_BOUNDS(jj >= 0 && jj < H && i >= 0 && i + 1 < W)) {
        const V t = *reinterpret_cast<const V*>(a + (int64_t)jj * ld + i);
        v[r][0] = t.x;
        v[r][1] = t.y;
      } else {
        v[r][0] = v[r][1] = (T)0;
      }
    } else {
      const bool row = jj >= 0 && jj < H;
      v[r][0] = (row && i >= 0 && i < W) ? a[(int64_t)jj * ld + i] : (T)0;
      v[r][1] = (row && i + 1 >= 0 && i + 1 < W) ? a[(int64_t)jj * ld + i + 1] : (T)0;
    }
  }
}

// Store the owned cells (rows [r_lo, r_hi) of the thread's RPT, both columns when owned).
template <typename T, int RPT, bool BOUNDED>
__device__ __forceinline__ void reg_store(const T (&v)[RPT][2], T* __restrict__ a, int64_t ld, int j, int i, int H,
                                          int W, bool cols_owned, int r_lo, int r_hi) {
  using V = typename Pair<T>::V;
  if (!cols_owned) return;
#pragma unroll
  for (int r = 0; r < RPT; ++r) {
    if (r < r_lo || r >= r_hi) continue;
    const int jj = j + r;
    if (!BOUNDED) {
      if (!SG_IN_BOUNDS(jj >= 0 && jj < H && i >= 0 && i + 1 < W)) continue;
      V t;
      t.x = v[r][0];
      t.y = v[r][1];
      *reinterpret_cast<V*>(a + (int64_t)jj * ld + i) = t;
    } else {
      if (jj >= H || !SG_IN_BOUNDS(jj >= 0 && i >= 0)) continue;
      if (i < W) a[(int64_t)jj * ld + i] = v[r][0];
      if (i + 1 < W) a[(int64_t)jj * ld + i + 1] = v[r][1];
    }
  }
}

template <typename T, int SW, int RPT, int NWARP>
struct RegPre {
  static constexpr int HALO = 2 * SW + 2;
  static constexpr int TXO = kRW - 2 * HALO;          // owned columns
  static constexpr int TYO = NWARP * RPT - 2 * HALO;  // owned rows
  static_assert(RPT % 2 == 0 && TYO > 0 && TXO > 0, "bad register tile");
};

template <typename T, int SW, int RPT, int NWARP>
struct RegPost {
  static constexpr int HALO = 2 * SW;
  static constexpr int TXO = kRW - 2 * HALO;
  static constexpr int TYO = NWARP * RPT - 2 * HALO;
  static_assert(RPT % 2 == 0 && TYO > 0 && TXO > 0, "bad register tile");
};

template <typename T, int SW, int RPT, int NWARP, bool BOUNDED>
__device__ __forceinline__ void reg_pre_body(RegXchg<T, NWARP>& x, const T* __restrict__ e_in, T* __restrict__ e_out,
                                             const T* __restrict__ bsrc, int64_t ld, int H, int W, T* __restrict__ bc,
                                             int64_t ldc, int Hc, int Wc, T omega, int i0, int j0,
                                             T* __restrict__ ec_zero = nullptr) {
  using S = RegPre<T, SW, RPT, NWARP>;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int i = i0 + 2 * lane, j = j0 + w * RPT;
  T e[RPT][2], b[RPT][2];
  reg_load<T, RPT, BOUNDED>(b, bsrc, ld, j, i, H, W);
  if (e_in) {
    reg_load<T, RPT, BOUNDED>(e, e_in, ld, j, i, H, W);
    reg_sweeps<T, RPT, NWARP, 2 * SW, 0, BOUNDED>(x, e, b, omega, w, lane, j, i, H, W);
  } else {
#pragma unroll
    for (int r = 0; r < RPT; ++r) e[r][0] = e[r][1] = (T)0;
    reg_first_half_sweep_from_zero<T, RPT, BOUNDED>(e, b, omega, j, i, H, W);
    reg_sweeps<T, RPT, NWARP, 2 * SW, 1, BOUNDED>(x, e, b, omega, w, lane, j, i, H, W);
  }
  // residual b - A e in place of b
  T above[2], below[2];
  exchange_rows<T, RPT, NWARP>(x, (2 * SW) & 1, e, w, lane, above, below);
#pragma unroll
  for (int r = 0; r < RPT; ++r) {
    const T l1 = shfl_up1(e[r][1]);
    const T r0 = shfl_down1(e[r][0]);
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const T xv = e[r][q];
      const T left = q == 0 ? l1 : e[r][0];
      const T right = q == 0 ? e[r][1] : r0;
      const T up = r > 0 ? e[r > 0 ? r - 1 : 0][q] : above[q];
      const T down = r < RPT - 1 ? e[r < RPT - 1 ? r + 1 : 0][q] : below[q];
      if (!BOUNDED) {
        if constexpr (sizeof(T) == 8)  // float64: the cheaper sum form (see the fused post kernel)
          b[r][q] = b[r][q] + (((left + right) + (up + down)) - (T)4 * xv);
        else
          b[r][q] = b[r][q] + (left - xv) + (right - xv) + (up - xv) + (down - xv);
      } else {
        const int jj = j + r, ii = i + q;
        T acc = (T)0;
        if (jj >= 0 && jj < H && ii >= 0 && ii < W) {
          acc = b[r][q];
          if (ii > 0) acc += left - xv;
          if (ii < W - 1) acc += right - xv;
          if (jj > 0) acc += up - xv;
          if (jj < H - 1) acc += down - xv;
        }
        b[r][q] = acc;
      }
    }
  }
  // full weighting along x: coarse column I = i0 / 2 + lane from fine columns 2I - 1 .. 2I + 2
  const int I = (i0 >> 1) + lane;
  T wx0 = (T)0.25, wx1 = (T)0.75, wx2 = (T)0.75, wx3 = (T)0.25;
  if (BOUNDED) {
    wx0 = (2 * I - 1 >= 0 && 2 * I - 1 < W) ? (T)w1(2 * I - 1, I, Wc) : (T)0;
    wx1 = (2 * I < W) ? (T)w1(2 * I, I, Wc) : (T)0;
    wx2 = (2 * I + 1 < W) ? (T)w1(2 * I + 1, I, Wc) : (T)0;
    wx3 = (2 * I + 2 < W) ? (T)w1(2 * I + 2, I, Wc) : (T)0;
  }
  T X[RPT];
#pragma unroll
  for (int r = 0; r < RPT; ++r) {
    const T rl = shfl_up1(b[r][1]);
    const T rr = shfl_down1(b[r][0]);
    T acc = (T)0;
    acc += wx0 * rl;
    acc += wx1 * b[r][0];
    acc += wx2 * b[r][1];
    acc += wx3 * rr;
    X[r] = acc;
  }
  x.xtop[w][lane] = X[0];
  x.xbot[w][lane] = X[RPT - 1];
  __syncthreads();
  const T xa = x.xbot[w > 0 ? w - 1 : w][lane];
  const T xb = x.xtop[w < NWARP - 1 ? w + 1 : w][lane];
  // along y: coarse row J = j / 2 + m from X rows 2m - 1 .. 2m + 2
  const bool cols_owned = 2 * lane >= S::HALO && 2 * lane < S::HALO + S::TXO && I < Wc;
  if (cols_owned) {
#pragma unroll
    for (int m = 0; m < RPT / 2; ++m) {
      const int rt = w * RPT + 2 * m;  // tile row of fine row 2J
      if (rt < S::HALO || rt >= S::HALO + S::TYO) continue;
      const int J = (j >> 1) + m;
      if (J >= Hc) continue;
      const T x0 = m > 0 ? X[m > 0 ? 2 * m - 1 : 0] : xa;
      const T x3 = 2 * m + 2 < RPT ? X[2 * m + 2 < RPT ? 2 * m + 2 : 0] : xb;
      T wy0 = (T)0.25, wy1 = (T)0.75, wy2 = (T)0.75, wy3 = (T)0.25;
      if (BOUNDED) {
        wy0 = (2 * J - 1 >= 0 && 2 * J - 1 < H) ? (T)w1(2 * J - 1, J, Hc) : (T)0;
        wy1 = (2 * J < H) ? (T)w1(2 * J, J, Hc) : (T)0;
        wy2 = (2 * J + 1 < H) ? (T)w1(2 * J + 1, J, Hc) : (T)0;
        wy3 = (2 * J + 2 < H) ? (T)w1(2 * J + 2, J, Hc) : (T)0;
      }
      T acc = (T)0;
      acc += wy0 * x0;
      acc += wy1 * X[2 * m];
      acc += wy2 * X[2 * m + 1];
      acc += wy3 * x3;
      bc[(int64_t)J * ldc + I] = acc;
      if (ec_zero) ec_zero[(int64_t)J * ldc + I] = (T)0;  // the coarse correction starts at 0
    }
  }
  const int r_lo = S::HALO - w * RPT, r_hi = S::HALO + S::TYO - w * RPT;
  reg_store<T, RPT, BOUNDED>(e, e_out, ld, j, i, H, W, 2 * lane >= S::HALO && 2 * lane < S::HALO + S::TXO, r_lo,
                             r_hi);
}

#ifndef SG_REGTILE_BODIES_ONLY
// pre: SW sweeps from e_in (NULL: zero initial guess), residual and its full weighting
// into bc; the smoothed cells go to e_out.
// b_alt (fine level of a fused solve only): the rhs alternates between b and b_alt from
// cycle to cycle (b on even cycles), as k_gmg_post_final_reg writes the next one.
template <typename T, int SW, int RPT, int NWARP, int MINB>
__global__ void __launch_bounds__(32 * NWARP, MINB) k_gmg_pre_reg(const T* __restrict__ e_in, T* __restrict__ e_out,
                                                           const T* __restrict__ b, const T* __restrict__ b_alt,
                                                           const GmgState* __restrict__ st, int64_t ld, int H, int W,
                                                           T* __restrict__ bc, int64_t ldc, int Hc, int Wc, T omega) {
  using S = RegPre<T, SW, RPT, NWARP>;
  __shared__ RegXchg<T, NWARP> x;
  if (b_alt && (st->cycles & 1)) b = b_alt;
  const int i0 = blockIdx.x * S::TXO - S::HALO;
  const int j0 = blockIdx.y * S::TYO - S::HALO;
  const bool inside = i0 >= 0 && i0 + kRW <= W && j0 >= 0 && j0 + NWARP * RPT <= H;
  if (inside)
    reg_pre_body<T, SW, RPT, NWARP, false>(x, e_in, e_out, b, ld, H, W, bc, ldc, Hc, Wc, omega, i0, j0);
  else
    reg_pre_body<T, SW, RPT, NWARP, true>(x, e_in, e_out, b, ld, H, W, bc, ldc, Hc, Wc, omega, i0, j0);
}
#endif

// e = e_in + P ec on the thread's cells, then SW sweeps (e and b stay in registers).
template <typename T, int SW, int RPT, int NWARP, bool BOUNDED>
__device__ __forceinline__ void reg_prolong_smooth(RegXchg<T, NWARP>& x, T (&e)[RPT][2], T (&b)[RPT][2],
                                                   const T* __restrict__ e_in, const T* __restrict__ bsrc, int64_t ld,
                                                   int H, int W, const T* __restrict__ ec, int64_t ldc, int Hc, int Wc,
                                                   T omega, int i0, int j0) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int i = i0 + 2 * lane, j = j0 + w * RPT;
  reg_load<T, RPT, BOUNDED>(b, bsrc, ld, j, i, H, W);
  reg_load<T, RPT, BOUNDED>(e, e_in, ld, j, i, H, W);
  // bilinear prolongation: fine (j, i) from coarse (J, I), (J, X), (Y, I), (Y, X) with
  // X = I -+ 1 for even / odd i and Y = J -+ 1 for even / odd j, both clamped to the level.
  // Every tile cell needs its exact start value (the sweeps only absorb wrong neighbours),
  // so the edge lanes load their outer coarse column instead of shuffling it in; with I
  // clamped on every lane, the shuffled neighbours are the clamped ones as well.
  const T w9 = (T)(9.0 / 16.0), w3 = (T)(3.0 / 16.0), wd = (T)(1.0 / 16.0);
  const int I = (i0 >> 1) + lane;
  const int Ic = I < 0 ? 0 : (I > Wc - 1 ? Wc - 1 : I);
  const int Iedge = lane == 0 ? (I - 1 < 0 ? 0 : (I - 1 > Wc - 1 ? Wc - 1 : I - 1))
                              : (I + 1 < 0 ? 0 : (I + 1 > Wc - 1 ? Wc - 1 : I + 1));
  const bool edge = lane == 0 || lane == 31;
  const int Jb = j >> 1;  // coarse row of the thread's first fine row (j even)
  auto fetch = [&](int J, T& cl, T& cm, T& cr) {
    const int Jc = J < 0 ? 0 : (J > Hc - 1 ? Hc - 1 : J);
    const T* row = ec + (int64_t)Jc * ldc;
    const bool ok = SG_IN_BOUNDS(Jc >= 0 && Jc < Hc && Ic >= 0 && Ic < Wc && Iedge >= 0 && Iedge < Wc);
    const T v = ok ? row[Ic] : (T)0;
    const T ve = (edge && ok) ? row[Iedge] : (T)0;
    const T lv = shfl_up1(v), rv = shfl_down1(v);
    cl = lane == 0 ? ve : lv;
    cm = v;
    cr = lane == 31 ? ve : rv;
  };
  T pl, pm, pr, cl, cm, cr;  // coarse rows Jb + m - 1 and Jb + m at columns I - 1, I, I + 1
  fetch(Jb - 1, pl, pm, pr);
  fetch(Jb, cl, cm, cr);
#pragma unroll
  for (int m = 0; m < RPT / 2; ++m) {
    T nl, nm, nr;
    fetch(Jb + m + 1, nl, nm, nr);
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int r = 2 * m + h;
      // fine row 2J (even): Y = J - 1; fine row 2J + 1 (odd): Y = J + 1
      const T yl = h == 0 ? pl : nl, ym = h == 0 ? pm : nm, yr = h == 0 ? pr : nr;
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        T acc = (T)0;
        acc += w9 * cm;
        acc += w3 * (q == 0 ? cl : cr);
        acc += w3 * ym;
        acc += wd * (q == 0 ? yl : yr);
        if (!BOUNDED || (j + r >= 0 && j + r < H && i + q >= 0 && i + q < W)) e[r][q] = e[r][q] + acc;
      }
    }
    pl = cl;
    pm = cm;
    pr = cr;
    cl = nl;
    cm = nm;
    cr = nr;
  }
  reg_sweeps<T, RPT, NWARP, 2 * SW, 0, BOUNDED>(x, e, b, omega, w, lane, j, i, H, W);
}

template <typename T, int SW, int RPT, int NWARP, bool BOUNDED>
__device__ __forceinline__ void reg_post_body(RegXchg<T, NWARP>& x, const T* __restrict__ e_in, T* __restrict__ e_out,
                                              const T* __restrict__ bsrc, int64_t ld, int H, int W,
                                              const T* __restrict__ ec, int64_t ldc, int Hc, int Wc, T omega, int i0,
                                              int j0) {
  using S = RegPost<T, SW, RPT, NWARP>;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int i = i0 + 2 * lane, j = j0 + w * RPT;
  T e[RPT][2], b[RPT][2];
  reg_prolong_smooth<T, SW, RPT, NWARP, BOUNDED>(x, e, b, e_in, bsrc, ld, H, W, ec, ldc, Hc, Wc, omega, i0, j0);
  const int r_lo = S::HALO - w * RPT, r_hi = S::HALO + S::TYO - w * RPT;
  reg_store<T, RPT, BOUNDED>(e, e_out, ld, j, i, H, W, 2 * lane >= S::HALO && 2 * lane < S::HALO + S::TXO, r_lo,
                             r_hi);
}

#ifndef SG_REGTILE_BODIES_ONLY
// post: e_out = smoothed (e_in + P ec).
template <typename T, int SW, int RPT, int NWARP, int MINB>
__global__ void __launch_bounds__(32 * NWARP, MINB) k_gmg_post_reg(const T* __restrict__ e_in, T* __restrict__ e_out,
                                                            const T* __restrict__ b, int64_t ld, int H, int W,
                                                            const T* __restrict__ ec, int64_t ldc, int Hc, int Wc,
                                                            T omega) {
  using S = RegPost<T, SW, RPT, NWARP>;
  __shared__ RegXchg<T, NWARP> x;
  const int i0 = blockIdx.x * S::TXO - S::HALO;
  const int j0 = blockIdx.y * S::TYO - S::HALO;
  const bool inside = i0 >= 0 && i0 + kRW <= W && j0 >= 0 && j0 + NWARP * RPT <= H;
  if (inside)
    reg_post_body<T, SW, RPT, NWARP, false>(x, e_in, e_out, b, ld, H, W, ec, ldc, Hc, Wc, omega, i0, j0);
  else
    reg_post_body<T, SW, RPT, NWARP, true>(x, e_in, e_out, b, ld, H, W, ec, ldc, Hc, Wc, omega, i0, j0);
}
#endif

__device__ __forceinline__ void prefetch_l2(const void* ptr) {
  asm volatile("prefetch.global.L2 [%0];" ::"l"(ptr));
}

// Fine level of a fused solve: post-smoothing, the correction p += e and the next residual
// in one pass. The residual follows r_new = r - A e (A p = sum over open faces of
// p - p_nb), which equals bf - A (p + e) up to rounding; every cell it writes needs e on
// its four neighbours only, so the tile halo is 2 SW + 2 (as for the pre kernel) and p is
// read and written on owned cells alone. The cycle rhs alternates between b0 and b1 by the
// parity of the cycle count (read from b0 on even cycles, next one written to the other).
// r64: the residual in the precision of p when it differs from the cycle's (mixed
// precision); otherwise the cycle rhs itself is the residual. Per-block sums of r^2 go to
// partial[] for k_gmg_finalize_rel.
template <typename TC, typename TP, int SW, int RPT, int NWARP, bool BOUNDED>
__device__ __forceinline__ void reg_post_final_body(RegXchg<TC, NWARP>& x, const TC* __restrict__ e_in,
                                                    const TC* __restrict__ bsrc, TC* __restrict__ bdst, int64_t ld,
                                                    int H, int W, const TC* __restrict__ ec, int64_t ldc, int Hc,
                                                    int Wc, TC omega, TP* __restrict__ p, int64_t ldp,
                                                    TP* __restrict__ r64, int i0, int j0, double& sq,
                                                    const FirstCycle& fc = FirstCycle{nullptr, 0, 0, 0, 0, 0.0, 0.0}) {
  using S = RegPre<TC, SW, RPT, NWARP>;
  // only mixed precision carries r64; the other instantiations compile without the first-cycle
  // path (which would cost them registers)
  const bool first = sizeof(TC) != sizeof(TP) && fc.active;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int i = i0 + 2 * lane, j = j0 + w * RPT;
  const bool cols_owned = 2 * lane >= S::HALO && 2 * lane < S::HALO + S::TXO && (!BOUNDED || i < W);
  const int r_lo = S::HALO - w * RPT, r_hi = S::HALO + S::TYO - w * RPT;
  // p and r64 are only needed after the sweeps: start bringing the owned rows into L2 now
  if (cols_owned && !first) {
#pragma unroll
    for (int r = 0; r < RPT; ++r) {
      if (r < r_lo || r >= r_hi || (BOUNDED && j + r >= H)) continue;
      prefetch_l2(p + (int64_t)(j + r) * ldp + i);
      if (r64) prefetch_l2(r64 + (int64_t)(j + r) * ld + i);
    }
  }
  TC e[RPT][2], b[RPT][2];
  reg_prolong_smooth<TC, SW, RPT, NWARP, BOUNDED>(x, e, b, e_in, bsrc, ld, H, W, ec, ldc, Hc, Wc, omega, i0, j0);
  TC above[2], below[2];
  exchange_rows<TC, RPT, NWARP>(x, (2 * SW) & 1, e, w, lane, above, below);
  using VC = typename Pair<TC>::V;
  using VP = typename Pair<TP>::V;
#pragma unroll
  for (int r = 0; r < RPT; ++r) {
    const TC l1 = shfl_up1(e[r][1]);
    const TC r0 = shfl_down1(e[r][0]);
    if (r < r_lo || r >= r_hi || !cols_owned) continue;
    const int jj = j + r;
    if (BOUNDED && jj >= H) continue;
    if (!SG_IN_BOUNDS(jj >= 0 && jj < H && i >= 0 && (BOUNDED || i + 1 < W))) continue;
    const int64_t o = (int64_t)jj * ld + i;
    TP acc[2];
    if (first && r64) {  // the first cycle's residual, from the divergence
#pragma unroll
      for (int q = 0; q < 2; ++q)
        acc[q] = (!BOUNDED || i + q < W) ? (TP)first_cycle_rhs(fc, (int64_t)jj * fc.ldd + i + q) : (TP)0;
    } else if (r64 && !BOUNDED) {
      const VP t = *reinterpret_cast<const VP*>(r64 + o);
      acc[0] = t.x;
      acc[1] = t.y;
    } else {
#pragma unroll
      for (int q = 0; q < 2; ++q) acc[q] = r64 ? ((!BOUNDED || i + q < W) ? r64[o + q] : (TP)0) : (TP)b[r][q];
    }
    TP xv[2];
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const int ii = i + q;
      xv[q] = (TP)e[r][q];
      const TP left = (TP)(q == 0 ? l1 : e[r][0]);
      const TP right = (TP)(q == 0 ? e[r][1] : r0);
      const TP up = (TP)(r > 0 ? e[r > 0 ? r - 1 : 0][q] : above[q]);
      const TP down = (TP)(r < RPT - 1 ? e[r < RPT - 1 ? r + 1 : 0][q] : below[q]);
      if (!BOUNDED) {
        if constexpr (sizeof(TP) == 8) {
          // float64: one sum and one fused multiply-add (the float32 form below keeps the
          // differences, which stay exact near convergence where the sum would cancel)
          acc[q] += ((left + right) + (up + down)) - (TP)4 * xv[q];
        } else {
          acc[q] += left - xv[q];
          acc[q] += right - xv[q];
          acc[q] += up - xv[q];
          acc[q] += down - xv[q];
        }
      } else {
        if (ii > 0) acc[q] += left - xv[q];
        if (ii < W - 1) acc[q] += right - xv[q];
        if (jj > 0) acc[q] += up - xv[q];
        if (jj < H - 1) acc[q] += down - xv[q];
      }
    }
    TP* pc = p + (int64_t)jj * ldp + i;
    if (!BOUNDED) {
      pc[0] = (first ? (TP)0 : pc[0]) + xv[0];
      pc[1] = (first ? (TP)0 : pc[1]) + xv[1];
      if (r64) {
        VP t;
        t.x = acc[0];
        t.y = acc[1];
        *reinterpret_cast<VP*>(r64 + o) = t;
      }
      VC c;
      c.x = (TC)acc[0];
      c.y = (TC)acc[1];
      *reinterpret_cast<VC*>(bdst + o) = c;
      sq += (double)acc[0] * (double)acc[0];
      sq += (double)acc[1] * (double)acc[1];
    } else {
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        if (i + q >= W) continue;
        pc[q] = (first ? (TP)0 : pc[q]) + xv[q];
        if (r64) r64[o + q] = acc[q];
        bdst[o + q] = (TC)acc[q];
        sq += (double)acc[q] * (double)acc[q];
      }
    }
  }
}

#ifndef SG_REGTILE_BODIES_ONLY
template <typename TC, typename TP, int SW, int RPT, int NWARP, int MINB>
__global__ void __launch_bounds__(32 * NWARP, MINB)
    k_gmg_post_final_reg(const TC* __restrict__ e_in, TC* __restrict__ b0, TC* __restrict__ b1,
                         const GmgState* __restrict__ st, int64_t ld, int H, int W, const TC* __restrict__ ec,
                         int64_t ldc, int Hc, int Wc, TC omega, TP* __restrict__ p, int64_t ldp, TP* __restrict__ r64,
                         double* __restrict__ partial, FirstCycle fc) {
  using S = RegPre<TC, SW, RPT, NWARP>;
  __shared__ RegXchg<TC, NWARP> x;
  const bool odd = st->cycles & 1;
  const TC* bsrc = odd ? b1 : b0;
  TC* bdst = odd ? b0 : b1;
  const int i0 = blockIdx.x * S::TXO - S::HALO;
  const int j0 = blockIdx.y * S::TYO - S::HALO;
  const bool inside = i0 >= 0 && i0 + kRW <= W && j0 >= 0 && j0 + NWARP * RPT <= H;
  double sq = 0.0;
  fc.active = sizeof(TC) != sizeof(TP) && fc.active && st->cycles == 0;
  fc.alpha = st->alpha;
  fc.mean = st->bmean;
  if (inside)
    reg_post_final_body<TC, TP, SW, RPT, NWARP, false>(x, e_in, bsrc, bdst, ld, H, W, ec, ldc, Hc, Wc, omega, p, ldp,
                                                      r64, i0, j0, sq, fc);
  else
    reg_post_final_body<TC, TP, SW, RPT, NWARP, true>(x, e_in, bsrc, bdst, ld, H, W, ec, ldc, Hc, Wc, omega, p, ldp,
                                                     r64, i0, j0, sq, fc);
  const double s = block_sum(sq);
  if (threadIdx.x == 0) partial[blockIdx.y * gridDim.x + blockIdx.x] = s;
}
#endif

// Rows per thread, warps per block and minimum resident blocks per SM of the register
// tiles (the last caps the registers a thread may use); MINB_FINAL for the fused fine-level
// post kernel.
#ifndef SG_REG_F32_RPT
#define SG_REG_F32_RPT 6
#define SG_REG_F32_NWARP 8
#define SG_REG_F32_MINB 4
#endif
#ifndef SG_REG_F64_RPT
#define SG_REG_F64_RPT 4
#define SG_REG_F64_NWARP 8
#define SG_REG_F64_MINB 4
#endif
#ifndef SG_REG_FINAL_MINB
#define SG_REG_FINAL_MINB 4
#endif
// the fused fine-level post kernel's rows per thread and warps (measured on B200: 6 x 8 for
// FP32 cycles, 4 x 8 for FP64, as for the level kernels)
#ifndef SG_REG_FINAL_F32_RPT
#define SG_REG_FINAL_F32_RPT 6
#define SG_REG_FINAL_F32_NWARP 8
#endif
#ifndef SG_REG_FINAL_F64_RPT
#define SG_REG_FINAL_F64_RPT SG_REG_F64_RPT
#define SG_REG_FINAL_F64_NWARP SG_REG_F64_NWARP
#endif
template <int R, int N, int M, int RF, int NF>
struct RegShapeOf {
  static constexpr int RPT = R, NWARP = N, MINB = M, MINB_FINAL = SG_REG_FINAL_MINB;
  static constexpr int RPT_FINAL = RF, NWARP_FINAL = NF;
};
template <typename T>
struct RegShape;
template <>
struct RegShape<float> : RegShapeOf<SG_REG_F32_RPT, SG_REG_F32_NWARP, SG_REG_F32_MINB, SG_REG_FINAL_F32_RPT,
                                    SG_REG_FINAL_F32_NWARP> {};
template <>
struct RegShape<double> : RegShapeOf<SG_REG_F64_RPT, SG_REG_F64_NWARP, SG_REG_F64_MINB, SG_REG_FINAL_F64_RPT,
                                     SG_REG_FINAL_F64_NWARP> {};
