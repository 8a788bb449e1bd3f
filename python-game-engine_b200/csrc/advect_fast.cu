// Semi-Lagrangian advection of float32 fields in float32 arithmetic
// (advection.py:112-180: the same backtrace, clamped bilinear sampling and masks).
//
// The reference evaluates positions and weights in float64 even for float32 fields, which
// on this GPU makes its faithful restatement (k_advect_uv / k_advect_scalar) wait on the
// conversion unit: every gathered value is widened and every position converted. Here the
// backtrace is kept relative to the sampling point's own cell: the offset o = -vel * dt / h
// is a small float32, floor(o) and the weight o - floor(o) are exact in float32 for |o| <
// 2^22, and the sample point's index is the integer cell index plus floor(o). The weights
// then carry float32's relative precision (not that of a float32 absolute position), and the
// interpolation is two float32 lerps; results differ from the reference's by rounding only
// (<= 1e-6 relative to the field's magnitude in the tests, inside the 1e-5 float32 bar).
//
// Clamping follows advection.py:31-38: indices are clamped to the grid before the weight is
// taken, so a sample whose bracket leaves the grid takes the edge value.
#include <algorithm>

#include "common.cuh"

namespace sg {

// Clamped bilinear sample of f (rows x cols, row stride ld; rows * ld < 2^31) at
// (bi + ox, bj + oy).
__device__ __forceinline__ float sample_rel(const float* __restrict__ f, int ld, int rows, int cols, int bi, int bj,
                                            float ox, float oy) {
  // keep the offsets finite and far from integer overflow (NaN ends at an edge, as in the
  // reference kernels' saturating conversions)
  ox = fminf(fmaxf(ox, -1048576.f), 1048576.f);
  oy = fminf(fmaxf(oy, -1048576.f), 1048576.f);
  const float fx = floorf(ox), fy = floorf(oy);
  const int x0 = bi + (int)fx, y0 = bj + (int)fy;
  if ((unsigned)x0 < (unsigned)(cols - 1) && (unsigned)y0 < (unsigned)(rows - 1)) {
    // the whole 2 x 2 stencil inside the grid (almost every sample): no clamping
    const float* r0 = f + y0 * ld + x0;
    const float tx = ox - fx, ty = oy - fy;
    const float a = r0[0], b = r0[1], cc = r0[ld], d = r0[ld + 1];
    const float c0 = fmaf(b - a, tx, a);
    const float c1 = fmaf(d - cc, tx, cc);
    return fmaf(c1 - c0, ty, c0);
  }
  const bool inx = x0 >= 0 && x0 < cols - 1;
  const bool iny = y0 >= 0 && y0 < rows - 1;
  const int xa = min(max(x0, 0), cols - 1), xb = inx ? x0 + 1 : xa;
  const int ya = min(max(y0, 0), rows - 1), yb = iny ? y0 + 1 : ya;
  const float tx = inx ? ox - fx : 0.f, ty = iny ? oy - fy : 0.f;
  const float* r0 = f + ya * ld;
  const float* r1 = f + yb * ld;
  const float c0 = fmaf(r0[xb] - r0[xa], tx, r0[xa]);
  const float c1 = fmaf(r1[xb] - r1[xa], tx, r1[xa]);
  return fmaf(c1 - c0, ty, c0);
}

// The mean of a 2 x 2 block (a b / c d) as two lerps at 1/2 and one between them, the
// bilinear sample at the block's centre without index arithmetic.
__device__ __forceinline__ float centre4(float a, float b, float c, float d) {
  const float c0 = fmaf(b - a, 0.5f, a);
  const float c1 = fmaf(d - c, 0.5f, c);
  return fmaf(c1 - c0, 0.5f, c0);
}

// u faces (H x (W+1)) and v faces ((H+1) x W) in one launch; c = dt / h.
template <int MM>
__global__ void k_advect_uv_f32(int H, int W, const float* __restrict__ us, int ldus, float* __restrict__ ud, int ldud,
                                const float* __restrict__ vs, int ldvs, float* __restrict__ vd, int ldvd, MasksT<MM> m,
                                float c) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
#pragma unroll
  for (int q = 0; q < kRows; ++q) {
    const int j = row_of(q);
    if (j < H && i <= W) {
      float out = 0.f;
      if (m.u(j, i)) {
        // advection.py:130-154: v at the u face (i, j + 0.5) is the v grid at (i - 0.5, j + 0.5):
        // the 2 x 2 block of columns i - 1, i and rows j, j + 1 away from the side walls
        const float uu = us[j * ldus + i];
        const float vv = (i >= 1 && i <= W - 1)
                             ? centre4(vs[j * ldvs + i - 1], vs[j * ldvs + i], vs[(j + 1) * ldvs + i - 1],
                                       vs[(j + 1) * ldvs + i])
                             : sample_rel(vs, ldvs, H + 1, W, i, j, -0.5f, 0.5f);
        out = sample_rel(us, ldus, H, W + 1, i, j, -uu * c, -vv * c);
      }
      ud[j * ldud + i] = out;
    }
    if (j <= H && i < W) {
      float out = 0.f;
      if (m.v(j, i)) {
        // advection.py:156-180: u at the v face (i + 0.5, j) is the u grid at (i + 0.5, j - 0.5):
        // the 2 x 2 block of columns i, i + 1 and rows j - 1, j away from the floor and ceiling
        const float uu = (j >= 1 && j <= H - 1)
                             ? centre4(us[(j - 1) * ldus + i], us[(j - 1) * ldus + i + 1], us[j * ldus + i],
                                       us[j * ldus + i + 1])
                             : sample_rel(us, ldus, H, W + 1, i, j, 0.5f, -0.5f);
        const float vv = vs[j * ldvs + i];
        out = sample_rel(vs, ldvs, H + 1, W, i, j, -uu * c, -vv * c);
      }
      vd[j * ldvd + i] = out;
    }
  }
}

// advection.py:112-128 (+ dissipation, simulation.py:232)
template <int MM>
__global__ void k_advect_scalar_f32(int H, int W, const float* __restrict__ src, int lds, float* __restrict__ dst,
                                    int ldd, const float* __restrict__ u, int ldu, const float* __restrict__ v, int ldv,
                                    MasksT<MM> m, float c, float diss) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= W) return;
#pragma unroll
  for (int q = 0; q < kRows; ++q) {
    const int j = row_of(q);
    if (j >= H) continue;
    float out = 0.f;
    if (m.fluid(j, i)) {
      // face velocities at the cell centre: u grid at (i + 0.5, j), v grid at (i, j + 0.5)
      const float ua = u[j * ldu + i], ub = u[j * ldu + i + 1];
      const float va = v[j * ldv + i], vb = v[(j + 1) * ldv + i];
      const float uu = fmaf(ub - ua, 0.5f, ua);
      const float vv = fmaf(vb - va, 0.5f, va);
      out = sample_rel(src, lds, H, W, i, j, -uu * c, -vv * c) * diss;
    }
    dst[j * ldd + i] = out;
  }
}

// ------------------------------------------------------------------ forces, float32 arithmetic
// forces.py:19-105 for float32 fields: buoyancy from the density averaged onto the v face
// (rows 0 and H - 1 take d[j], row H gets no density term) and from the temperature (ambient
// where there is none), added as v += dt (b + t). The reference forms both terms in float64
// and rounds each to float32 before the sum; here they are float32 products throughout.
// A thread takes kForceRows consecutive faces of one column and loads each density row once.
constexpr int kForceRows = 8;
__global__ void k_apply_forces_f32(int H, int W, float* __restrict__ v, int ldv, const float* __restrict__ d, int ldd,
                                   const float* __restrict__ t, int ldt, float dt, float kd, float kt, float amb) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j0 = (blockIdx.y * blockDim.y + threadIdx.y) * kForceRows;
  if (i >= W || j0 > H) return;
  // density rows j0 - 1 .. j0 + kForceRows - 1 (inside the grid) and the v faces, all loaded first
  float dr[kForceRows + 1], vv[kForceRows];
#pragma unroll
  for (int q = 0; q <= kForceRows; ++q) {
    const int j = j0 - 1 + q;
    dr[q] = (j >= 0 && j < H) ? d[j * ldd + i] : 0.f;
  }
#pragma unroll
  for (int q = 0; q < kForceRows; ++q) vv[q] = (j0 + q <= H) ? v[(j0 + q) * ldv + i] : 0.f;
#pragma unroll
  for (int q = 0; q < kForceRows; ++q) {
    const int j = j0 + q;
    if (j > H) break;
    float bf = 0.f;
    if (j < H) {
      const float dd = (j == 0 || j == H - 1) ? dr[q + 1] : 0.5f * (dr[q] + dr[q + 1]);
      bf = kd * dd;  // kd = -density_coefficient * gravity
    }
    float tt = amb;
    if (t) tt = j == 0 ? t[i] : (j == H ? t[(H - 1) * ldt + i] : 0.5f * (t[(j - 1) * ldt + i] + t[j * ldt + i]));
    const float tf = kt * (tt - amb);  // kt = -buoyancy_coefficient
    v[j * ldv + i] = fmaf(dt, bf + tf, vv[q]);
  }
}

// ------------------------------------------------------------------ projection tail, float32 arithmetic
// The substep's tail (pressure_gradient.py:4-37, boundaries.py:7-39, then divergence.py:4-25
// and residual.py:6-42 on the projected field) as k_project_metrics walks it -- a warp owns 32
// columns and walks kTailRowsF rows, each face projected once -- with float32 arithmetic in
// place of the reference's float64 intermediates.
#ifndef SG_TAIL_ROWS_F32
#define SG_TAIL_ROWS_F32 4
#endif
constexpr int kTailRowsF = SG_TAIL_ROWS_F32;

template <typename MK, int SM>
__device__ __forceinline__ float proj_u_f32(int j, int i, int H, int W, float uk, float pc, float pn, const MK& m,
                                            int solid_mode, const uint8_t* __restrict__ solid, int64_t lds,
                                            float scale) {
  if ((i > 0 && solid_at_t<SM>(solid_mode, solid, lds, H, W, j, i - 1)) ||
      (i < W && solid_at_t<SM>(solid_mode, solid, lds, H, W, j, i)))
    return 0.f;
  return (m.u(j, i) && i > 0 && i < W) ? fmaf(-scale, pc - pn, uk) : 0.f;
}

template <typename MK, int SM>
__device__ __forceinline__ float proj_v_f32(int j, int i, int H, int W, float vk, float pc, float pn, const MK& m,
                                            int solid_mode, const uint8_t* __restrict__ solid, int64_t lds,
                                            float scale) {
  if ((j > 0 && solid_at_t<SM>(solid_mode, solid, lds, H, W, j - 1, i)) ||
      (j < H && solid_at_t<SM>(solid_mode, solid, lds, H, W, j, i)))
    return 0.f;
  return (m.v(j, i) && j > 0 && j < H) ? fmaf(-scale, pc - pn, vk) : 0.f;
}

template <int MM, int SM>
__global__ void __launch_bounds__(kBX * kBY) k_project_metrics_f32(
    int H, int W, const float* __restrict__ ui, int ldui, const float* __restrict__ vi, int ldvi, float* __restrict__ uo,
    int lduo, float* __restrict__ vo, int ldvo, const float* __restrict__ p, int ldp, MasksT<MM> m, int solid_mode,
    const uint8_t* __restrict__ solid, int64_t lds, float scale, float* __restrict__ div, int ldd, float inv,
    float alpha, float beta, float* __restrict__ res, int ldr) {
  using MK = MasksT<MM>;
  const int lane = threadIdx.x;  // blockDim.x == 32: a warp is one row segment
  const int i = blockIdx.x * kBX + lane;
  const int j0 = (blockIdx.y * kBY + threadIdx.y) * kTailRowsF;
  if (j0 >= H) return;  // uniform over the warp
  const bool cell = i < W, ucol = i <= W;
  const float* pc_col = p + i;
  float p_dn = (cell && j0 > 0) ? pc_col[(j0 - 1) * ldp] : 0.f;
  float p_c = cell ? pc_col[j0 * ldp] : 0.f;
  float v_lo = 0.f;
  if (cell) {
    v_lo = proj_v_f32<MK, SM>(j0, i, H, W, vi[j0 * ldvi + i], p_c, p_dn, m, solid_mode, solid, lds, scale);
    if (j0 == 0) vo[i] = v_lo;
  }
  // the strip's pressure, u and v rows, loaded before any of them is used
  float pr[kTailRowsF], ur_in[kTailRowsF], vr_in[kTailRowsF];
#pragma unroll
  for (int q = 0; q < kTailRowsF; ++q) {
    const int j = j0 + q;
    pr[q] = (cell && j + 1 < H) ? pc_col[(j + 1) * ldp] : 0.f;
    ur_in[q] = (ucol && j < H) ? ui[j * ldui + i] : 0.f;
    vr_in[q] = (cell && j < H) ? vi[(j + 1) * ldvi + i] : 0.f;
  }
#pragma unroll
  for (int q = 0; q < kTailRowsF; ++q) {
    const int j = j0 + q;
    if (j >= H) break;  // uniform over the warp
    const float p_up = pr[q];
    const float uin = ur_in[q];
    const float vin = vr_in[q];
    float p_l = __shfl_up_sync(0xffffffffu, p_c, 1);
    float p_r = __shfl_down_sync(0xffffffffu, p_c, 1);
    if (lane == 0) p_l = (i > 0 && i - 1 < W) ? pc_col[j * ldp - 1] : 0.f;
    if (lane == kBX - 1) p_r = (i + 1 < W) ? pc_col[j * ldp + 1] : 0.f;
    float ul = 0.f;
    if (ucol) {
      ul = proj_u_f32<MK, SM>(j, i, H, W, uin, p_c, p_l, m, solid_mode, solid, lds, scale);
      uo[j * lduo + i] = ul;
    }
    float ur = __shfl_down_sync(0xffffffffu, ul, 1);
    if (lane == kBX - 1 && i + 1 <= W)
      ur = proj_u_f32<MK, SM>(j, i + 1, H, W, ui[j * ldui + i + 1], p_r, p_c, m, solid_mode, solid, lds, scale);
    if (cell) {
      const float v_hi = proj_v_f32<MK, SM>(j + 1, i, H, W, vin, p_up, p_c, m, solid_mode, solid, lds, scale);
      vo[(j + 1) * ldvo + i] = v_hi;
      // divergence.py:4-25 on the projected faces
      const float du = (m.u(j, i + 1) ? ur : 0.f) - (m.u(j, i) ? ul : 0.f);
      const float dv = (m.v(j + 1, i) ? v_hi : 0.f) - (m.v(j, i) ? v_lo : 0.f);
      const float dval = (du + dv) * inv;
      div[j * ldd + i] = dval;
      // residual.py:6-42: neighbours behind closed faces (or outside) take the cell's value
      float r = 0.f;
      if (m.fluid(j, i)) {
        const float l = m.u(j, i) ? (i > 0 ? p_l : p_c) : p_c;
        const float rr = m.u(j, i + 1) ? (i < W - 1 ? p_r : p_c) : p_c;
        const float dn = m.v(j, i) ? (j > 0 ? p_dn : p_c) : p_c;
        const float up = m.v(j + 1, i) ? (j < H - 1 ? p_up : p_c) : p_c;
        const float sum = ((l + rr) + dn) + up;
        r = fmaf(-beta, p_c, fmaf(alpha, dval, sum));
      }
      res[j * ldr + i] = r;
      v_lo = v_hi;
    }
    p_dn = p_c;
    p_c = p_up;
  }
}

}  // namespace sg

using namespace sg;

extern "C" {

int sg_apply_forces_f32(int64_t H, int64_t W, void* v, int64_t ld_v, const void* density, int64_t ld_d,
                        const void* temperature, int64_t ld_t, double dt, double gravity, double buoyancy_coefficient,
                        double density_coefficient, double ambient_temperature, void* stream) {
  SG_REQUIRE(H >= 1 && W >= 1 && H <= (1 << 28) && W <= (1 << 28), "bad grid %lld x %lld", (long long)H, (long long)W);
  SG_REQUIRE(v && density, "null field pointer");
  SG_REQUIRE(ld_v >= W && ld_d >= W && (!temperature || ld_t >= W), "row stride below row length");
  SG_REQUIRE((H + 1) * std::max(std::max(ld_v, ld_d), temperature ? ld_t : (int64_t)0) < ((int64_t)1 << 31),
             "fields of 2^31 elements or more: use sg_apply_forces");
  const dim3 gf((unsigned)((W + kBX - 1) / kBX), (unsigned)((H + 1 + kBY * kForceRows - 1) / (kBY * kForceRows)));
  SG_LAUNCH(k_apply_forces_f32<<<gf, block2d(), 0, as_stream(stream)>>>(
      (int)H, (int)W, (float*)v, (int)ld_v, (const float*)density, (int)ld_d, (const float*)temperature, (int)ld_t,
      (float)dt, (float)(-density_coefficient * gravity), (float)(-buoyancy_coefficient), (float)ambient_temperature));
  return check_launch("sg_apply_forces_f32");
}

int sg_project_metrics_f32(int64_t H, int64_t W, const void* u_in, int64_t ld_ui, const void* v_in, int64_t ld_vi,
                           void* u_out, int64_t ld_uo, void* v_out, int64_t ld_vo, const void* p, int64_t ld_p,
                           int mask_mode, const uint8_t* fmu, int64_t ld_fmu, const uint8_t* fmv, int64_t ld_fmv,
                           const uint8_t* is_fluid, int64_t ld_fluid, int solid_mode, const uint8_t* solid,
                           int64_t ld_s, double fluid_density, double cell_size, double dt, double alpha,
                           double reciprocal_beta, void* div, int64_t ld_div, void* res, int64_t ld_res,
                           void* stream) {
  SG_REQUIRE(H >= 1 && W >= 1 && H <= (1 << 28) && W <= (1 << 28), "bad grid %lld x %lld", (long long)H, (long long)W);
  SG_REQUIRE(u_in && v_in && u_out && v_out && p && div && res, "null field pointer");
  SG_REQUIRE(u_in != u_out && v_in != v_out, "the projection here is out of place");
  SG_REQUIRE(ld_ui >= W + 1 && ld_vi >= W && ld_uo >= W + 1 && ld_vo >= W && ld_p >= W && ld_div >= W && ld_res >= W,
             "row stride below row length");
  SG_REQUIRE(fluid_density != 0.0 && cell_size > 0.0 && reciprocal_beta != 0.0, "bad coefficients");
  SG_REQUIRE(mask_mode == SG_MASK_OPEN || mask_mode == SG_MASK_RING || (mask_mode == SG_MASK_PLANES && fmu && fmv),
             "bad mask mode or missing mask planes");
  SG_REQUIRE(mask_mode != SG_MASK_PLANES || is_fluid, "is_fluid plane required");
  SG_REQUIRE(solid_mode == SG_MASK_NONE || solid_mode == SG_MASK_RING || (solid_mode == SG_MASK_PLANES && solid),
             "bad solid mode or missing solid plane");
  const int64_t ldmax = std::max(std::max(std::max(ld_ui, ld_vi), std::max(ld_uo, ld_vo)),
                                 std::max(ld_p, std::max(ld_div, ld_res)));
  SG_REQUIRE((H + 1) * ldmax < ((int64_t)1 << 31), "fields of 2^31 elements or more: use sg_project_metrics");
  Masks m = make_masks(mask_mode, H, W, fmu, ld_fmu, fmv, ld_fmv, is_fluid, ld_fluid);
  const float scale = (float)(dt / (fluid_density * cell_size));
  SG_MASK_DISPATCH(mask_mode, {
    SG_SOLID_DISPATCH(solid_mode, {
      SG_LAUNCH(k_project_metrics_f32<MM, SM><<<dim3((unsigned)((W + 1 + kBX - 1) / kBX),
                                                     (unsigned)((H + kBY * kTailRowsF - 1) / (kBY * kTailRowsF))),
                                                block2d(), 0, as_stream(stream)>>>(
          (int)H, (int)W, (const float*)u_in, (int)ld_ui, (const float*)v_in, (int)ld_vi, (float*)u_out, (int)ld_uo,
          (float*)v_out, (int)ld_vo, (const float*)p, (int)ld_p, m.as<MM>(), solid_mode, solid, ld_s, scale,
          (float*)div, (int)ld_div, (float)(1.0 / cell_size), (float)alpha, (float)(1.0 / reciprocal_beta),
          (float*)res, (int)ld_res));
    });
  });
  return check_launch("sg_project_metrics_f32");
}

int sg_advect_velocity_f32(int64_t H, int64_t W, const void* u_src, int64_t ld_us, void* u_dst, int64_t ld_ud,
                           const void* v_src, int64_t ld_vs, void* v_dst, int64_t ld_vd, int mask_mode,
                           const uint8_t* fmu, int64_t ld_fmu, const uint8_t* fmv, int64_t ld_fmv, double dt,
                           double cell_size, void* stream) {
  SG_REQUIRE(H >= 1 && W >= 1 && H <= (1 << 28) && W <= (1 << 28), "bad grid %lld x %lld", (long long)H, (long long)W);
  SG_REQUIRE(u_src && u_dst && v_src && v_dst, "null field pointer");
  SG_REQUIRE(ld_us >= W + 1 && ld_ud >= W + 1 && ld_vs >= W && ld_vd >= W, "row stride below row length");
  SG_REQUIRE(cell_size > 0.0, "cell_size must be positive");
  SG_REQUIRE(mask_mode == SG_MASK_OPEN || mask_mode == SG_MASK_RING || (mask_mode == SG_MASK_PLANES && fmu && fmv),
             "bad mask mode or missing mask planes");
  SG_REQUIRE((H + 1) * std::max(std::max(ld_us, ld_ud), std::max(ld_vs, ld_vd)) < ((int64_t)1 << 31),
             "fields of 2^31 elements or more: use sg_advect_velocity");
  Masks m = make_masks(mask_mode, H, W, fmu, ld_fmu, fmv, ld_fmv, nullptr, 0);
  const float c = (float)(dt / cell_size);
  SG_MASK_DISPATCH(mask_mode, {
    SG_LAUNCH(k_advect_uv_f32<MM><<<grid2d_rows(W + 1, H + 1), block2d(), 0, as_stream(stream)>>>(
        (int)H, (int)W, (const float*)u_src, (int)ld_us, (float*)u_dst, (int)ld_ud, (const float*)v_src, (int)ld_vs,
        (float*)v_dst, (int)ld_vd, m.as<MM>(), c));
  });
  return check_launch("sg_advect_velocity_f32");
}

int sg_advect_scalar_f32(int64_t H, int64_t W, const void* src, int64_t ld_src, void* dst, int64_t ld_dst,
                         const void* u, int64_t ld_u, const void* v, int64_t ld_v, int mask_mode,
                         const uint8_t* is_fluid, int64_t ld_fluid, double dt, double cell_size, double dissipation,
                         void* stream) {
  SG_REQUIRE(H >= 1 && W >= 1 && H <= (1 << 28) && W <= (1 << 28), "bad grid %lld x %lld", (long long)H, (long long)W);
  SG_REQUIRE(src && dst && u && v, "null field pointer");
  SG_REQUIRE(ld_src >= W && ld_dst >= W && ld_u >= W + 1 && ld_v >= W, "row stride below row length");
  SG_REQUIRE(cell_size > 0.0, "cell_size must be positive");
  SG_REQUIRE(mask_mode == SG_MASK_OPEN || mask_mode == SG_MASK_RING || (mask_mode == SG_MASK_PLANES && is_fluid),
             "bad mask mode or missing is_fluid plane");
  SG_REQUIRE((H + 1) * std::max(std::max(ld_src, ld_dst), std::max(ld_u, ld_v)) < ((int64_t)1 << 31),
             "fields of 2^31 elements or more: use sg_advect_scalar");
  Masks m = make_masks(mask_mode, H, W, nullptr, 0, nullptr, 0, is_fluid, ld_fluid);
  const float c = (float)(dt / cell_size);
  SG_MASK_DISPATCH(mask_mode, {
    SG_LAUNCH(k_advect_scalar_f32<MM><<<grid2d_rows(W, H), block2d(), 0, as_stream(stream)>>>(
        (int)H, (int)W, (const float*)src, (int)ld_src, (float*)dst, (int)ld_dst, (const float*)u, (int)ld_u,
        (const float*)v, (int)ld_v, m.as<MM>(), c, (float)dissipation));
  });
  return check_launch("sg_advect_scalar_f32");
}

}  // extern "C"

SG_BOUNDS_ACCESSOR(advect_fast)
