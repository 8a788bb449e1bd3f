// Single-block tail of the convergent multigrid for open-box levels (included by gmg.cu
// inside namespace sg; uses w1, rcp_open, warp_sum and kMaxLevels from there).
//
// When every level from the tail's first one down to the coarsest is an open box, one
// block of 1024 threads runs the whole rest of the cycle in shared memory: the levels up
// to 16 cells a side (measured best on B200: at 32^2 and 64^2 one SM's issue rate makes
// the block slower than two 16 x 16-tiled launches per level) cost a few barriers each
// here. Each level keeps
//   e: two colour planes of (H + 2) x (Wh + 2) (Wh = ceil(W / 2)), cell (j, i) of colour
//      c = (i + j) & 1 at plane c, row j + 1, column (i >> 1) + 1; the ring and the
//      slot past an odd row end stay 0, so out-of-grid neighbours read 0;
//   b: two colour planes of H x Wh.
// A half sweep then streams one plane and reads the other without bank conflicts, and
// the relaxation sum needs no bounds checks (a 0 neighbour adds nothing; only the
// neighbour count depends on the position). The cycle (V or W) runs as a loop over levels
// with a bit mask recording which W-cycle levels already made their first coarse visit.
#pragma once

#ifndef SG_OPEN_TAIL_MAX_SIDE
#define SG_OPEN_TAIL_MAX_SIDE 16
#endif
constexpr int kOpenTailMaxSide = SG_OPEN_TAIL_MAX_SIDE;
#ifndef SG_OPEN_TAIL_THREADS
#define SG_OPEN_TAIL_THREADS 1024
#endif
constexpr int kOpenTailThreads = SG_OPEN_TAIL_THREADS;
constexpr int kOTY = kOpenTailThreads / 32;  // block rows (threads are 32 x kOTY)

template <typename T>
struct OpenTailArgs {
  int n;                   // tail levels; the last one is the coarsest (exact solve)
  int H[kMaxLevels], W[kMaxLevels];
  int off_e[kMaxLevels];   // shared-memory offsets (elements of T) of the e planes
  int off_b[kMaxLevels];   // and of the b planes
  int e_total;             // elements of all e planes (zeroed at start)
  int off_x;               // restriction scratch: H x ceil(W / 2) of the first level
  int off_r;               // residual / correction scratch: H x W of the first level
  T* ge;                   // first tail level in global memory (e in/out, b in)
  const T* gb;
  int64_t gld;
  const double* pinv;      // coarsest pseudo-inverse
  T omega;
  int pre, post, wcycle, zero_init;
};

template <typename T>
struct OpenLevel {
  T* e;  // plane 0 at e, plane 1 at e + (H + 2) * P
  T* b;  // plane 0 at b, plane 1 at b + H * Wh
  int H, W, Wh, P;
  __device__ __forceinline__ T* ep(int c) const { return e + c * (H + 2) * P + P + 1; }
  __device__ __forceinline__ T* bp(int c) const { return b + c * H * Wh; }
  // (j, i) may lie one cell outside the grid (reads 0 there)
  __device__ __forceinline__ T& E(int j, int i) const { return ep((i + j) & 1)[j * P + (i >> 1)]; }
  __device__ __forceinline__ T& B(int j, int i) const { return bp((i + j) & 1)[j * Wh + (i >> 1)]; }
};

struct OpenTailTable {
  int H[kMaxLevels], W[kMaxLevels], off_e[kMaxLevels], off_b[kMaxLevels];
};

template <typename T>
__device__ __forceinline__ OpenLevel<T> open_level(const OpenTailTable& t, T* sm, int k) {
  OpenLevel<T> L;
  L.H = t.H[k];
  L.W = t.W[k];
  L.Wh = (L.W + 1) >> 1;
  L.P = L.Wh + 2;
  L.e = sm + t.off_e[k];
  L.b = sm + t.off_b[k];
  return L;
}

// Half sweep of colour c.
template <typename T>
__device__ void open_relax(const OpenLevel<T>& L, int c, T omega) {
  const int tx = threadIdx.x, ty = threadIdx.y;
  for (int j = ty; j < L.H; j += kOTY) {
    const int p = (c + j) & 1;  // colour-c cells of row j sit at columns i = 2k + p
    T* E = L.ep(c) + j * L.P;
    const T* O = L.ep(1 - c) + j * L.P;
    const T* Bc = L.bp(c) + j * L.Wh;
    for (int k = tx; k < L.Wh; k += 32) {
      const int i = 2 * k + p;
      if (i >= L.W) continue;
      const int n = 4 - (i == 0) - (i == L.W - 1) - (j == 0) - (j == L.H - 1);
      if (n <= 0) continue;
      const T acc = Bc[k] + O[k + p - 1] + O[k + p] + O[k - L.P] + O[k + L.P];
      const T x = E[k];
      E[k] = x + omega * (acc * rcp_open<T>(n) - x);
    }
  }
  __syncthreads();
}

// bc = P^T (b - A e) and ec = 0, in three passes over shared memory: the residual of every
// fine cell into R (H x W, natural order), its full weighting along x into X (H x Wc),
// then along y into the coarse planes. Interior columns / rows use the constant weights
// (1, 3, 3, 1) / 4; the outermost ones take theirs from w1.
template <typename T>
__device__ void open_restrict(const OpenLevel<T>& L, const OpenLevel<T>& C, T* R, T* X) {
  const int tx = threadIdx.x, ty = threadIdx.y;
#pragma unroll
  for (int c = 0; c < 2; ++c)
    for (int j = ty; j < L.H; j += kOTY) {
      const int p = (c + j) & 1;
      const T* E = L.ep(c) + j * L.P;
      const T* O = L.ep(1 - c) + j * L.P;
      const T* Bc = L.bp(c) + j * L.Wh;
      for (int k = tx; k < L.Wh; k += 32) {
        const int i = 2 * k + p;
        if (i >= L.W) continue;
        const int n = 4 - (i == 0) - (i == L.W - 1) - (j == 0) - (j == L.H - 1);
        const T x = E[k];
        const T s = O[k + p - 1] + O[k + p] + O[k - L.P] + O[k + L.P];
        R[j * L.W + i] = Bc[k] + (s - (T)n * x);
      }
    }
  __syncthreads();
  for (int j = ty; j < L.H; j += kOTY) {
    const T* Rj = R + j * L.W;
    for (int I = tx; I < C.W; I += 32) {
      T acc = (T)0;
      if (I >= 1 && 2 * I + 2 < L.W && I + 1 < C.W - 1) {
        acc += (T)0.25 * Rj[2 * I - 1];
        acc += (T)0.75 * Rj[2 * I];
        acc += (T)0.75 * Rj[2 * I + 1];
        acc += (T)0.25 * Rj[2 * I + 2];
      } else {
#pragma unroll
        for (int d = 0; d < 4; ++d) {
          const int i = 2 * I - 1 + d;
          if (i < 0 || i >= L.W) continue;
          const T w = (T)w1(i, I, C.W);
          if (w != (T)0) acc += w * Rj[i];
        }
      }
      X[j * C.W + I] = acc;
    }
  }
  __syncthreads();
  for (int J = ty; J < C.H; J += kOTY)
    for (int I = tx; I < C.W; I += 32) {
      T acc = (T)0;
      if (J >= 1 && 2 * J + 2 < L.H && J + 1 < C.H - 1) {
        acc += (T)0.25 * X[(2 * J - 1) * C.W + I];
        acc += (T)0.75 * X[(2 * J) * C.W + I];
        acc += (T)0.75 * X[(2 * J + 1) * C.W + I];
        acc += (T)0.25 * X[(2 * J + 2) * C.W + I];
      } else {
#pragma unroll
        for (int d = 0; d < 4; ++d) {
          const int j = 2 * J - 1 + d;
          if (j < 0 || j >= L.H) continue;
          const T w = (T)w1(j, J, C.H);
          if (w != (T)0) acc += w * X[j * C.W + I];
        }
      }
      C.B(J, I) = acc;
      C.E(J, I) = (T)0;
    }
  __syncthreads();
}

// e += P ec (bilinear, clamped at the level's edges): the coarse correction is first
// copied to natural order in R (Hc x Wc), then every fine plane is updated in place.
template <typename T>
__device__ void open_prolong(const OpenLevel<T>& C, const OpenLevel<T>& L, T* R) {
  const T w9 = (T)(9.0 / 16.0), w3 = (T)(3.0 / 16.0), wd = (T)(1.0 / 16.0);
  const int tx = threadIdx.x, ty = threadIdx.y;
  for (int J = ty; J < C.H; J += kOTY)
    for (int I = tx; I < C.W; I += 32) R[J * C.W + I] = C.E(J, I);
  __syncthreads();
#pragma unroll
  for (int c = 0; c < 2; ++c)
    for (int j = ty; j < L.H; j += kOTY) {
      const int p = (c + j) & 1;
      const int J = j >> 1;
      int Y = J + ((j & 1) ? 1 : -1);
      Y = Y < 0 ? 0 : (Y > C.H - 1 ? C.H - 1 : Y);
      const T* c0 = R + J * C.W;
      const T* c1 = R + Y * C.W;
      T* E = L.ep(c) + j * L.P;
      for (int k = tx; k < L.Wh; k += 32) {
        const int i = 2 * k + p;
        if (i >= L.W) continue;
        const int I = i >> 1;
        int Xc = I + ((i & 1) ? 1 : -1);
        Xc = Xc < 0 ? 0 : (Xc > C.W - 1 ? C.W - 1 : Xc);
        T acc = (T)0;
        acc += w9 * c0[I];
        acc += w3 * c0[Xc];
        acc += w3 * c1[I];
        acc += wd * c1[Xc];
        E[k] += acc;
      }
    }
  __syncthreads();
}

// e = pinv b on the coarsest level (natural cell order q = j W + i), one row per warp.
template <typename T>
__device__ void open_coarse_solve(const OpenLevel<T>& L, const double* __restrict__ pinv) {
  const int n = L.H * L.W;
  const int tid = threadIdx.y * 32 + threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int row = warp; row < n; row += kOpenTailThreads / 32) {
    double acc = 0.0;
    for (int q = lane; q < n; q += 32) {
      const int j = q / L.W, i = q - j * L.W;
      acc += pinv[(int64_t)row * n + q] * (double)L.B(j, i);
    }
    acc = warp_sum(acc);
    if (lane == 0) {
      const int j = row / L.W, i = row - j * L.W;
      L.E(j, i) = (T)acc;
    }
  }
  __syncthreads();
}

template <typename T>
__global__ void __launch_bounds__(kOpenTailThreads) k_gmg_tail_open(const __grid_constant__ OpenTailArgs<T> a) {
  extern __shared__ __align__(16) unsigned char open_tail_smem[];
  T* sm = reinterpret_cast<T*>(open_tail_smem);
  __shared__ OpenTailTable tab;
  const int tid = threadIdx.y * 32 + threadIdx.x;
  if (tid < a.n) {
    tab.H[tid] = a.H[tid];
    tab.W[tid] = a.W[tid];
    tab.off_e[tid] = a.off_e[tid];
    tab.off_b[tid] = a.off_b[tid];
  }
  for (int q = tid; q < a.e_total; q += kOpenTailThreads) sm[q] = (T)0;
  __syncthreads();
  {
    const OpenLevel<T> L0 = open_level(tab, sm, 0);
    for (int j = threadIdx.y; j < L0.H; j += kOTY)
      for (int i = threadIdx.x; i < L0.W; i += 32) {
        L0.B(j, i) = a.gb[(int64_t)j * a.gld + i];
        if (!a.zero_init) L0.E(j, i) = a.ge[(int64_t)j * a.gld + i];
      }
  }
  __syncthreads();
  T* X = sm + a.off_x;
  T* R = sm + a.off_r;
  const int last = a.n - 1;
  int k = 0;
  bool enter = true;
  unsigned second = 0;  // bit k: level k already sent its first visit to level k + 1
  while (true) {
    if (enter) {
      const OpenLevel<T> L = open_level(tab, sm, k);
      if (k == last) {
        open_coarse_solve(L, a.pinv);
        if (k == 0) break;
        --k;
        enter = false;
        continue;
      }
      for (int s = 0; s < a.pre; ++s) {
        open_relax(L, 0, a.omega);
        open_relax(L, 1, a.omega);
      }
      open_restrict(L, open_level(tab, sm, k + 1), R, X);
      second &= ~(1u << k);
      ++k;
      continue;
    }
    // back on level k from level k + 1
    if (a.wcycle && k + 1 < last && !((second >> k) & 1u)) {
      second |= 1u << k;
      ++k;
      enter = true;
      continue;
    }
    const OpenLevel<T> L = open_level(tab, sm, k);
    open_prolong(open_level(tab, sm, k + 1), L, R);
    for (int s = 0; s < a.post; ++s) {
      open_relax(L, 0, a.omega);
      open_relax(L, 1, a.omega);
    }
    if (k == 0) break;
    --k;
  }
  {
    const OpenLevel<T> L0 = open_level(tab, sm, 0);
    for (int j = threadIdx.y; j < L0.H; j += kOTY)
      for (int i = threadIdx.x; i < L0.W; i += 32) a.ge[(int64_t)j * a.gld + i] = L0.E(j, i);
  }
}
