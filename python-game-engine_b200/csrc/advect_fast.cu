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

}  // namespace sg

using namespace sg;

extern "C" {

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
