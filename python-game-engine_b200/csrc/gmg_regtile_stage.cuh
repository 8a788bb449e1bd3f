// The fused fine-level post kernel with its fine-precision operands staged in shared memory
// (included inside namespace sg by gmg.cu after gmg_regtile.cuh; uses bulk_copy.cuh).
//
// k_gmg_post_final_reg reads p and the carried residual r64 (32 of its 45 bytes per cell in
// mixed precision) only after the sweeps, and brings them towards the SM with an L2 prefetch.
// Here, on tiles that lie inside the grid, threads 0 .. 2 TYO - 1 each issue one bulk copy of
// an owned row of p or r64 straight into shared memory when the block starts, so the transfer
// runs under the prolongation and the sweeps without registers or issue slots, and the final
// phase reads shared memory. Edge tiles take the unstaged body. The arithmetic is that of
// k_gmg_post_final_reg, so both kernels write the same bits.
#pragma once

template <typename TP, int TXO, int TYO>
struct StagedPR {
  TP p[TYO * TXO];
  TP r[TYO * TXO];
  uint64_t bar;
};

template <typename TC, typename TP, int SW, int RPT, int NWARP>
__device__ __forceinline__ void reg_post_final_body_staged(RegXchg<TC, NWARP>& x,
                                                           StagedPR<TP, RegPre<TC, SW, RPT, NWARP>::TXO,
                                                                    RegPre<TC, SW, RPT, NWARP>::TYO>& sp,
                                                           const TC* __restrict__ e_in, const TC* __restrict__ bsrc,
                                                           TC* __restrict__ bdst, int64_t ld, int H, int W,
                                                           const TC* __restrict__ ec, int64_t ldc, int Hc, int Wc,
                                                           TC omega, TP* __restrict__ p, int64_t ldp,
                                                           TP* __restrict__ r64, int i0, int j0, double& sq, bool& ok,
                                                           const FirstCycle& fc, bool staged_any) {
  using S = RegPre<TC, SW, RPT, NWARP>;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int i = i0 + 2 * lane, j = j0 + w * RPT;
  const bool cols_owned = 2 * lane >= S::HALO && 2 * lane < S::HALO + S::TXO;
  const int r_lo = S::HALO - w * RPT, r_hi = S::HALO + S::TYO - w * RPT;
  TC e[RPT][2], b[RPT][2];
  reg_prolong_smooth<TC, SW, RPT, NWARP, false>(x, e, b, e_in, bsrc, ld, H, W, ec, ldc, Hc, Wc, omega, i0, j0);
  TC above[2], below[2];
  exchange_rows<TC, RPT, NWARP>(x, (2 * SW) & 1, e, w, lane, above, below);
  // every thread waits, so the block cannot retire while a copy is still landing
  if (staged_any && !mbar_wait(&sp.bar, 0)) ok = false;
  using VC = typename Pair<TC>::V;
  using VP = typename Pair<TP>::V;
  const int cs = 2 * lane - S::HALO;  // the thread's first column in the staged rows
#pragma unroll
  for (int r = 0; r < RPT; ++r) {
    const TC l1 = shfl_up1(e[r][1]);
    const TC r0 = shfl_down1(e[r][0]);
    if (r < r_lo || r >= r_hi || !cols_owned) continue;
    const int jj = j + r;
    const int k = w * RPT + r - S::HALO;  // staged row
    if (!SG_IN_BOUNDS(jj >= 0 && jj < H && i >= 0 && i + 1 < W && k >= 0 && k < S::TYO && cs >= 0 &&
                      cs + 1 < S::TXO))
      continue;
    const int64_t o = (int64_t)jj * ld + i;
    TP acc[2];
    if (sizeof(TC) != sizeof(TP) && fc.active && r64) {  // the first cycle's r64, from the staged divergence
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const int64_t so = (int64_t)k * S::TXO + cs + q;
        const double d = fc.f64 ? reinterpret_cast<const double*>(sp.p)[so]
                                : (double)reinterpret_cast<const float*>(sp.p)[so];
        double x2 = fc.alpha * d;
        if (fc.sub_mean) x2 -= fc.mean;
        acc[q] = (TP)x2;
      }
    } else if (r64) {
      const VP t = *reinterpret_cast<const VP*>(sp.r + k * S::TXO + cs);
      acc[0] = t.x;
      acc[1] = t.y;
    } else {
      acc[0] = (TP)b[r][0];
      acc[1] = (TP)b[r][1];
    }
    TP xv[2];
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      xv[q] = (TP)e[r][q];
      const TP left = (TP)(q == 0 ? l1 : e[r][0]);
      const TP right = (TP)(q == 0 ? e[r][1] : r0);
      const TP up = (TP)(r > 0 ? e[r > 0 ? r - 1 : 0][q] : above[q]);
      const TP down = (TP)(r < RPT - 1 ? e[r < RPT - 1 ? r + 1 : 0][q] : below[q]);
      if constexpr (sizeof(TP) == 8) {
        acc[q] += ((left + right) + (up + down)) - (TP)4 * xv[q];
      } else {
        acc[q] += left - xv[q];
        acc[q] += right - xv[q];
        acc[q] += up - xv[q];
        acc[q] += down - xv[q];
      }
    }
    VP pv;
    if (sizeof(TC) != sizeof(TP) && fc.active) {  // p is 0 on a solve's first cycle from a zero guess
      pv.x = (TP)0;
      pv.y = (TP)0;
    } else {
      pv = *reinterpret_cast<const VP*>(sp.p + k * S::TXO + cs);
    }
    VP pn;
    pn.x = pv.x + xv[0];
    pn.y = pv.y + xv[1];
    *reinterpret_cast<VP*>(p + (int64_t)jj * ldp + i) = pn;
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
  }
}

#ifndef SG_REGTILE_BODIES_ONLY
// Same arguments as k_gmg_post_final_reg (st writable: a bounded wait that gives up sets
// st->dev_error). The host chooses this kernel only when p, ldp, r64 and ld put every staged
// row on 16-byte boundaries.
template <typename TC, typename TP, int SW, int RPT, int NWARP, int MINB>
__global__ void __launch_bounds__(32 * NWARP, MINB)
    k_gmg_post_final_stage(const TC* __restrict__ e_in, TC* __restrict__ b0, TC* __restrict__ b1,
                           GmgState* __restrict__ st, int64_t ld, int H, int W, const TC* __restrict__ ec,
                           int64_t ldc, int Hc, int Wc, TC omega, TP* __restrict__ p, int64_t ldp,
                           TP* __restrict__ r64, double* __restrict__ partial, FirstCycle fc) {
  using S = RegPre<TC, SW, RPT, NWARP>;
  static_assert((S::TXO * sizeof(TP)) % 16 == 0, "staged rows must be whole 16-byte units");
  static_assert(2 * S::TYO <= 32 * NWARP, "one thread per staged row");
  __shared__ RegXchg<TC, NWARP> x;
  __shared__ __align__(16) StagedPR<TP, S::TXO, S::TYO> sp;
  const bool odd = st->cycles & 1;
  const TC* bsrc = odd ? b1 : b0;
  TC* bdst = odd ? b0 : b1;
  const int i0 = blockIdx.x * S::TXO - S::HALO;
  const int j0 = blockIdx.y * S::TYO - S::HALO;
  const bool inside = i0 >= 0 && i0 + kRW <= W && j0 >= 0 && j0 + NWARP * RPT <= H;
  double sq = 0.0;
  // the first cycle of a solve from a zero guess (mixed precision only: the others carry no r64)
  fc.active = sizeof(TC) != sizeof(TP) && fc.active && st->cycles == 0;
  fc.alpha = st->alpha;
  fc.mean = st->bmean;
  if (inside) {
    const int t = threadIdx.x;
    // rows to stage: p and r64 (or p alone); on the first cycle only the divergence rows that
    // form r64 (p is 0), or nothing without r64
    const int nrow = fc.active ? (r64 ? S::TYO : 0) : (r64 ? 2 * S::TYO : S::TYO);
    if (nrow > 0) {
      if (t == 0) {
        mbar_init(&sp.bar, 1);
        mbar_fence_init();
      }
      __syncthreads();
      constexpr uint32_t kRowBytes = S::TXO * sizeof(TP);
      const uint32_t div_bytes = (uint32_t)S::TXO * (fc.f64 ? 8u : 4u);
      if (t == 0) mbar_arrive_expect_tx(&sp.bar, (uint32_t)nrow * (fc.active ? div_bytes : kRowBytes));
      if (t < nrow) {
        const int k = t < S::TYO ? t : t - S::TYO;
        const int64_t jj = j0 + S::HALO + k, ii = i0 + S::HALO;
        if (fc.active)
          bulk_g2s(reinterpret_cast<unsigned char*>(sp.p) + (size_t)k * div_bytes,
                   reinterpret_cast<const unsigned char*>(fc.div) + (jj * fc.ldd + ii) * (fc.f64 ? 8 : 4), div_bytes,
                   &sp.bar);
        else if (t < S::TYO)
          bulk_g2s(sp.p + k * S::TXO, p + jj * ldp + ii, kRowBytes, &sp.bar);
        else
          bulk_g2s(sp.r + k * S::TXO, r64 + jj * ld + ii, kRowBytes, &sp.bar);
      }
    }
    bool ok = true;
    reg_post_final_body_staged<TC, TP, SW, RPT, NWARP>(x, sp, e_in, bsrc, bdst, ld, H, W, ec, ldc, Hc, Wc, omega, p,
                                                       ldp, r64, i0, j0, sq, ok, fc, nrow > 0);
    if (!ok) atomicExch(&st->dev_error, kDevErrBulkWait);
  } else {
    reg_post_final_body<TC, TP, SW, RPT, NWARP, true>(x, e_in, bsrc, bdst, ld, H, W, ec, ldc, Hc, Wc, omega, p, ldp,
                                                     r64, i0, j0, sq, fc);
  }
  const double s = block_sum(sq);
  if (threadIdx.x == 0) partial[blockIdx.y * gridDim.x + blockIdx.x] = s;
}
#endif
