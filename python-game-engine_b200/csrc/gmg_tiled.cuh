// Fused tiled level kernels of the convergent multigrid (included by gmg.cu and batch.cu
// inside namespace sg; uses w1 and rcp_open of gmg_weights.cuh).
//
// For open-box levels (every cell fluid, every interior face open) one launch runs a whole
// side of a cycle on a tile of fine cells held in shared memory (64 x 32 on large levels,
// 16 x 16 on levels too small to fill the GPU with large tiles):
//   pre:  SW red-black sweeps, the residual and its full-weighting restriction; reads e
//         (not at all for a zero initial guess) and b once, writes e and the coarse rhs;
//   post: bilinear prolongation of the coarse correction plus SW sweeps.
// The tile carries a halo that shrinks by one ring per half sweep, so every cell it writes
// gets exactly the value a sequence of grid-wide half sweeps would give it. A launch reads
// e from one buffer and writes another (pre: E0 or nothing -> E1, post: E1 -> E0), so no
// block reads halo cells another block of the same launch is writing.
// In shared memory the tile is kept in checkerboard-split layout: smem cell (r, c) is fine
// cell (j0 + r, i0 + c), has colour (par0 + r + c) & 1 and lives at
// plane[colour][r][c >> 1], so a half sweep streams one colour plane and reads the other
// without bank conflicts. Tiles whose whole halo lies inside the grid ("interior" tiles,
// all but the outermost) take a path without bounds checks (every cell has 4 neighbours).
#pragma once

constexpr int kTX = 64, kTY = 32;   // fine cells of a large-level tile
constexpr int kSX = 16, kSY = 16;   // fine cells of a small-level tile (more blocks per level)
constexpr int kTBX = 32, kTBY = 8;  // threads of a tile block
constexpr int kTThreads = kTBX * kTBY;

template <typename T>
struct SplitTile {
  T* e;  // 2 colour planes of EY x EXh
  T* b;
  int EXh, EY, par0, i0, j0, H, W;
  __device__ __forceinline__ int colour(int r, int c) const { return (par0 + r + c) & 1; }
  __device__ __forceinline__ T* ep(int col) const { return e + col * EY * EXh; }
  __device__ __forceinline__ T* bp(int col) const { return b + col * EY * EXh; }
  __device__ __forceinline__ T& E(int r, int c) const { return ep(colour(r, c))[r * EXh + (c >> 1)]; }
  __device__ __forceinline__ T& B(int r, int c) const { return bp(colour(r, c))[r * EXh + (c >> 1)]; }
};

__device__ __forceinline__ int tile_tid() { return threadIdx.y * kTBX + threadIdx.x; }
// threads of the block: kTThreads, or more on levels with few tiles (shorter phases)
__device__ __forceinline__ int tile_nt() { return kTBX * blockDim.y; }

// Relax the cells of colour col in the tile grown by RING rings (smem rows/cols
// [HALO - RING, HALO + TY|TX + RING)); every neighbour is inside the loaded tile.
template <typename T, bool INTERIOR, int HALO, int RING, int EXh, int TX, int TY>
__device__ __forceinline__ void relax_ring(const SplitTile<T>& t, int col, T omega) {
  constexpr int RLO = HALO - RING, NR = TY + 2 * RING;
  constexpr int CLO = HALO - RING, CHI = HALO + TX + RING;
  constexpr int KW = (CHI - CLO + 1) / 2;  // cells of one colour per row, upper bound
  constexpr int N = NR * KW;
  T* E = t.ep(col);
  const T* Bc = t.bp(col);
  const T* O = t.ep(1 - col);
  for (int f = tile_tid(); f < N; f += tile_nt()) {
    const int rr = f / KW;
    const int r = RLO + rr;
    const int p = (col + t.par0 + r) & 1;  // columns of colour col in this row: c = p + 2k
    const int k = ((CLO - p + 1) >> 1) + (f - rr * KW);
    if (p + 2 * k >= CHI) continue;
    const int o = r * EXh + k;
    if (INTERIOR) {
      const T acc = Bc[o] + O[o + p - 1] + O[o + p] + O[o - EXh] + O[o + EXh];
      const T x = E[o];
      E[o] = x + omega * (acc * (T)0.25 - x);
    } else {
      const int j = t.j0 + r, i = t.i0 + p + 2 * k;
      if (j < 0 || j >= t.H || i < 0 || i >= t.W) continue;
      T acc = Bc[o];
      int n = 0;
      if (i > 0) { acc += O[o + p - 1]; ++n; }
      if (i < t.W - 1) { acc += O[o + p]; ++n; }
      if (j > 0) { acc += O[o - EXh]; ++n; }
      if (j < t.H - 1) { acc += O[o + EXh]; ++n; }
      if (n == 0) continue;
      const T x = E[o];
      E[o] = x + omega * (acc * rcp_open<T>(n) - x);
    }
  }
}

// The first half sweep (colour 0, ring HALO - 1) from e = 0: every neighbour is 0, so a
// cell's update is omega * (b / n) (the general formula with x = 0 and a zero neighbour sum).
template <typename T, bool INTERIOR, int HALO, int EXh, int TX, int TY>
__device__ __forceinline__ void relax_first_from_zero(const SplitTile<T>& t, T omega) {
  constexpr int RING = HALO - 1;
  constexpr int RLO = HALO - RING, NR = TY + 2 * RING;
  constexpr int CLO = HALO - RING, CHI = HALO + TX + RING;
  constexpr int KW = (CHI - CLO + 1) / 2;
  constexpr int N = NR * KW;
  T* E = t.ep(0);
  const T* Bc = t.bp(0);
  for (int f = tile_tid(); f < N; f += tile_nt()) {
    const int rr = f / KW;
    const int r = RLO + rr;
    const int p = (t.par0 + r) & 1;
    const int k = ((CLO - p + 1) >> 1) + (f - rr * KW);
    if (p + 2 * k >= CHI) continue;
    const int o = r * EXh + k;
    if (INTERIOR) {
      E[o] = omega * (Bc[o] * (T)0.25);
    } else {
      const int j = t.j0 + r, i = t.i0 + p + 2 * k;
      if (j < 0 || j >= t.H || i < 0 || i >= t.W) continue;
      const int n = (i > 0) + (i < t.W - 1) + (j > 0) + (j < t.H - 1);
      if (n == 0) continue;
      E[o] = omega * (Bc[o] * rcp_open<T>(n));
    }
  }
}

// Half sweeps HS .. NHS-1 (colour = HS & 1, ring HALO - 1 - HS).
template <typename T, bool INTERIOR, int HALO, int EXh, int TX, int TY, int HS, int NHS>
__device__ __forceinline__ void relax_all(const SplitTile<T>& t, T omega) {
  if constexpr (HS < NHS) {
    relax_ring<T, INTERIOR, HALO, HALO - 1 - HS, EXh, TX, TY>(t, HS & 1, omega);
    __syncthreads();
    relax_all<T, INTERIOR, HALO, EXh, TX, TY, HS + 1, NHS>(t, omega);
  }
}

template <typename T, bool INTERIOR, int EX, int EY>
__device__ __forceinline__ void tile_load(const SplitTile<T>& t, const T* __restrict__ e, const T* __restrict__ b,
                                          int64_t ld) {
  for (int f = tile_tid(); f < EX * EY; f += tile_nt()) {
    const int r = f / EX, c = f - r * EX;
    const int j = t.j0 + r, i = t.i0 + c;
    const bool in = (INTERIOR && SG_IN_BOUNDS(j >= 0 && j < t.H && i >= 0 && i < t.W)) ||
                    (!INTERIOR && j >= 0 && j < t.H && i >= 0 && i < t.W);
    const int64_t g = (int64_t)j * ld + i;
    t.E(r, c) = (in && e) ? e[g] : (T)0;
    t.B(r, c) = in ? b[g] : (T)0;
  }
}

template <typename T, bool INTERIOR, int HALO, int TX, int TY>
__device__ __forceinline__ void tile_store(const SplitTile<T>& t, T* __restrict__ e, int64_t ld) {
  for (int f = tile_tid(); f < TX * TY; f += tile_nt()) {
    const int rr = f / TX, cc = f - rr * TX;
    const int j = t.j0 + HALO + rr, i = t.i0 + HALO + cc;
    if (INTERIOR ? SG_IN_BOUNDS(j >= 0 && j < t.H && i >= 0 && i < t.W) : (j < t.H && i < t.W))
      e[(int64_t)j * ld + i] = t.E(HALO + rr, HALO + cc);
  }
}

template <typename T, bool INTERIOR>
__device__ __forceinline__ T tile_residual(const SplitTile<T>& t, int r, int c) {
  const T x = t.E(r, c);
  if (INTERIOR) return t.B(r, c) + (t.E(r, c - 1) - x) + (t.E(r, c + 1) - x) + (t.E(r - 1, c) - x) + (t.E(r + 1, c) - x);
  const int j = t.j0 + r, i = t.i0 + c;
  if (j < 0 || j >= t.H || i < 0 || i >= t.W) return (T)0;
  T acc = t.B(r, c);
  if (i > 0) acc += t.E(r, c - 1) - x;
  if (i < t.W - 1) acc += t.E(r, c + 1) - x;
  if (j > 0) acc += t.E(r - 1, c) - x;
  if (j < t.H - 1) acc += t.E(r + 1, c) - x;
  return acc;
}

template <int SW, int TX, int TY>
struct PreShape {
  static constexpr int HALO = 2 * SW + 2;  // 2SW half sweeps + residual ring + restriction window
  static constexpr int EX = TX + 2 * HALO, EY = TY + 2 * HALO, EXh = EX / 2;
  static constexpr int XR = TY + 2, XC = TX / 2;
  template <typename T>
  static constexpr size_t bytes() { return (size_t)(4 * EY * EXh + XR * XC) * sizeof(T); }
};

template <int SW, int TX, int TY>
struct PostShape {
  static constexpr int HALO = 2 * SW;
  static constexpr int EX = TX + 2 * HALO, EY = TY + 2 * HALO, EXh = EX / 2;
  template <typename T>
  static constexpr size_t bytes() { return (size_t)(4 * EY * EXh) * sizeof(T); }
};

// (bx, by): the tile's position in the level's grid of TX x TY tiles.
template <typename T, int TX, int TY>
__device__ __forceinline__ SplitTile<T> make_tile(unsigned char* smem, int halo, int EXh, int EY, int H, int W, int bx,
                                                  int by) {
  SplitTile<T> t;
  T* base = reinterpret_cast<T*>(smem);
  t.e = base;
  t.b = base + 2 * EY * EXh;
  t.EXh = EXh;
  t.EY = EY;
  t.i0 = bx * TX - halo;
  t.j0 = by * TY - halo;
  t.par0 = (t.i0 + t.j0) & 1;
  t.H = H;
  t.W = W;
  return t;
}

template <typename T, int SW, int TX, int TY, bool INTERIOR>
__device__ __forceinline__ void pre_body(const SplitTile<T>& t, const T* __restrict__ e_in, T* __restrict__ e_out,
                                         const T* __restrict__ b, int64_t ld, T* __restrict__ bc, int64_t ldc, int Hc,
                                         int Wc, T omega, T* X, int bx, int by) {
  using S = PreShape<SW, TX, TY>;
  tile_load<T, INTERIOR, S::EX, S::EY>(t, e_in, b, ld);
  __syncthreads();
  if (e_in) {
    relax_all<T, INTERIOR, S::HALO, S::EXh, TX, TY, 0, 2 * SW>(t, omega);
  } else {
    relax_first_from_zero<T, INTERIOR, S::HALO, S::EXh, TX, TY>(t, omega);
    __syncthreads();
    relax_all<T, INTERIOR, S::HALO, S::EXh, TX, TY, 1, 2 * SW>(t, omega);
  }
  // residual on the tile plus one ring, in place of b (each cell reads only its own b)
  constexpr int RW = TX + 2, RH = TY + 2, LO = S::HALO - 1;
  for (int f = tile_tid(); f < RW * RH; f += tile_nt()) {
    const int rr = f / RW, cc = f - rr * RW;
    const T res = tile_residual<T, INTERIOR>(t, LO + rr, LO + cc);
    t.B(LO + rr, LO + cc) = res;
  }
  __syncthreads();
  // full weighting along x: X[rr][I'] over fine rows of the tile plus one ring
  const int H = t.H, W = t.W;
  for (int f = tile_tid(); f < S::XR * S::XC; f += tile_nt()) {
    const int rr = f / S::XC, Ip = f - rr * S::XC;
    const int I = bx * S::XC + Ip;
    T acc = (T)0;
    if (I < Wc) {
#pragma unroll
      for (int d = 0; d < 4; ++d) {
        const int i = 2 * I - 1 + d;
        if (i < 0 || i >= W) continue;
        const T w = (T)w1(i, I, Wc);
        if (w != (T)0) acc += w * t.B(LO + rr, 2 * Ip + LO + d);
      }
    }
    X[f] = acc;
  }
  __syncthreads();
  // along y
  for (int f = tile_tid(); f < (TY / 2) * S::XC; f += tile_nt()) {
    const int Jp = f / S::XC, Ip = f - Jp * S::XC;
    const int J = by * (TY / 2) + Jp, I = bx * S::XC + Ip;
    if (J >= Hc || I >= Wc) continue;
    T acc = (T)0;
#pragma unroll
    for (int d = 0; d < 4; ++d) {
      const int j = 2 * J - 1 + d;
      if (j < 0 || j >= H) continue;
      const T w = (T)w1(j, J, Hc);
      if (w != (T)0) acc += w * X[(2 * Jp + d) * S::XC + Ip];
    }
    bc[(int64_t)J * ldc + I] = acc;
  }
  tile_store<T, INTERIOR, S::HALO, TX, TY>(t, e_out, ld);
}

// pre: SW sweeps from e_in (NULL: zero initial guess) + residual + full weighting into
// bc (coarse tile TX/2 x TY/2); the smoothed tile goes to e_out.
template <typename T, int SW, int TX, int TY>
__global__ void __launch_bounds__(1024) k_gmg_pre_tiled(const T* __restrict__ e_in, T* __restrict__ e_out,
                                                             const T* __restrict__ b, int64_t ld, int H, int W,
                                                             T* __restrict__ bc, int64_t ldc, int Hc, int Wc, T omega) {
  using S = PreShape<SW, TX, TY>;
  extern __shared__ __align__(16) unsigned char smem[];
  SplitTile<T> t = make_tile<T, TX, TY>(smem, S::HALO, S::EXh, S::EY, H, W, blockIdx.x, blockIdx.y);
  T* X = reinterpret_cast<T*>(smem) + 4 * S::EY * S::EXh;
  const bool interior = t.i0 >= 0 && t.i0 + S::EX <= W && t.j0 >= 0 && t.j0 + S::EY <= H;
  if (interior)
    pre_body<T, SW, TX, TY, true>(t, e_in, e_out, b, ld, bc, ldc, Hc, Wc, omega, X, blockIdx.x, blockIdx.y);
  else
    pre_body<T, SW, TX, TY, false>(t, e_in, e_out, b, ld, bc, ldc, Hc, Wc, omega, X, blockIdx.x, blockIdx.y);
}

template <typename T, int SW, int TX, int TY, bool INTERIOR>
__device__ __forceinline__ void post_body(const SplitTile<T>& t, const T* __restrict__ e_in, T* __restrict__ e_out,
                                          const T* __restrict__ b, int64_t ld, const T* __restrict__ ec, int64_t ldc,
                                          int Hc, int Wc, T omega) {
  using S = PostShape<SW, TX, TY>;
  const T w9 = (T)(9.0 / 16.0), w3 = (T)(3.0 / 16.0), wd = (T)(1.0 / 16.0);
  for (int f = tile_tid(); f < S::EX * S::EY; f += tile_nt()) {
    const int r = f / S::EX, c = f - r * S::EX;
    const int j = t.j0 + r, i = t.i0 + c;
    T ev = (T)0, bv = (T)0;
    if (INTERIOR ? SG_IN_BOUNDS(j >= 0 && j < t.H && i >= 0 && i < t.W && (j >> 1) < Hc && (i >> 1) < Wc)
                 : (j >= 0 && j < t.H && i >= 0 && i < t.W)) {
      const int J = j >> 1, I = i >> 1;
      int Y = J + ((j & 1) ? 1 : -1), X = I + ((i & 1) ? 1 : -1);
      Y = Y < 0 ? 0 : (Y > Hc - 1 ? Hc - 1 : Y);
      X = X < 0 ? 0 : (X > Wc - 1 ? Wc - 1 : X);
      const T* c0 = ec + (int64_t)J * ldc;
      const T* c1 = ec + (int64_t)Y * ldc;
      T acc = (T)0;
      acc += w9 * c0[I];
      acc += w3 * c0[X];
      acc += w3 * c1[I];
      acc += wd * c1[X];
      const int64_t g = (int64_t)j * ld + i;
      ev = e_in[g] + acc;
      bv = b[g];
    }
    t.E(r, c) = ev;
    t.B(r, c) = bv;
  }
  __syncthreads();
  relax_all<T, INTERIOR, S::HALO, S::EXh, TX, TY, 0, 2 * SW>(t, omega);
  tile_store<T, INTERIOR, S::HALO, TX, TY>(t, e_out, ld);
}

// post: e_out = smoothed (e_in + P ec).
template <typename T, int SW, int TX, int TY>
__global__ void __launch_bounds__(1024) k_gmg_post_tiled(const T* __restrict__ e_in, T* __restrict__ e_out,
                                                              const T* __restrict__ b, int64_t ld, int H, int W,
                                                              const T* __restrict__ ec, int64_t ldc, int Hc, int Wc,
                                                              T omega) {
  using S = PostShape<SW, TX, TY>;
  extern __shared__ __align__(16) unsigned char smem[];
  SplitTile<T> t = make_tile<T, TX, TY>(smem, S::HALO, S::EXh, S::EY, H, W, blockIdx.x, blockIdx.y);
  const bool interior = t.i0 >= 0 && t.i0 + S::EX <= W && t.j0 >= 0 && t.j0 + S::EY <= H;
  if (interior)
    post_body<T, SW, TX, TY, true>(t, e_in, e_out, b, ld, ec, ldc, Hc, Wc, omega);
  else
    post_body<T, SW, TX, TY, false>(t, e_in, e_out, b, ld, ec, ldc, Hc, Wc, omega);
}
