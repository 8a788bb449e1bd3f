// Adjoint (reverse-mode) kernels of the smoke step, for gradients of a loss on the final
// state with respect to the initial state and to a per-step control force.
//
// The forward step is the one of simulation.py:186-265 with a control force added after the
// forces: plume sources (overwrite) -> buoyancy + control -> velocity self-advection ->
// density advection with the advected velocity (and dissipation) -> divergence ->
// pressure solve -> gradient subtraction and boundary zeroing. Every stage but the solve and
// the two advections is linear with fixed coefficients; its adjoint is the transpose.
// Semi-Lagrangian advection, value(x) = bilinear sample of the source at the backtraced
// point x = centre - vel * dt / h, is linear in the source (adjoint: the transpose of the
// interpolation, a scatter of lambda * weight into the four sampled cells) and depends on
// the velocity through x (adjoint: lambda * d sample / d x * (-dt / h), carried back through
// the fixed interpolation that produced the velocity at the centre). The sampling follows
// the reference exactly (advection.py:6-49: corner indices floor / ceil clamped to the
// grid, weights taken after clamping), so the derivative of a sample whose two corners
// coincide (clamped, or an exact integer coordinate) is 0 along that axis, as the forward
// function is flat there. The transpose of the density interpolation comes in two forms: an
// atomicAdd scatter, and a deterministic gather in which every source cell sums, in a fixed
// order, the weights that the stored backtrace stencils of the targets around it give it.
// The pressure solve's adjoint is the same symmetric solve (run by the caller).

#include "common.cuh"

namespace sg {

// Corner indices and weights of the reference's bilinear sample (see sample_ref).
struct Stencil {
  int x0, x1, y0, y1;
  double tx, ty;
};

__device__ __forceinline__ Stencil stencil_ref(int64_t rows, int64_t cols, double x, double y) {
  const int nc = (int)cols - 1, nr = (int)rows - 1;
  Stencil s;
  s.x0 = min(max(__double2int_rd(x), 0), nc);
  s.x1 = min(max(__double2int_ru(x), 0), nc);
  s.y0 = min(max(__double2int_rd(y), 0), nr);
  s.y1 = min(max(__double2int_ru(y), 0), nr);
  s.tx = x - (double)s.x0;
  s.ty = y - (double)s.y0;
  return s;
}

// The sample's value, rounded as sample_ref rounds it (corner differences in T).
template <typename T>
__device__ __forceinline__ double stencil_value(const T* __restrict__ f, int64_t ld, const Stencil& s) {
  const T c00 = f[(int64_t)s.y0 * ld + s.x0], c10 = f[(int64_t)s.y0 * ld + s.x1];
  const T c01 = f[(int64_t)s.y1 * ld + s.x0], c11 = f[(int64_t)s.y1 * ld + s.x1];
  const double c0 = lerp_ref(c00, c10, s.tx), c1 = lerp_ref(c01, c11, s.tx);
  return c0 + (c1 - c0) * s.ty;
}

// d sample / dx and d sample / dy.
template <typename T>
__device__ __forceinline__ void stencil_grad(const T* __restrict__ f, int64_t ld, const Stencil& s, double& gx,
                                             double& gy) {
  const T c00 = f[(int64_t)s.y0 * ld + s.x0], c10 = f[(int64_t)s.y0 * ld + s.x1];
  const T c01 = f[(int64_t)s.y1 * ld + s.x0], c11 = f[(int64_t)s.y1 * ld + s.x1];
  const T d0 = c10 - c00, d1 = c11 - c01;
  gx = (double)d0 * (1.0 - s.ty) + (double)d1 * s.ty;
  gy = lerp_ref(c01, c11, s.tx) - lerp_ref(c00, c10, s.tx);
}

// lam_f[corners] += lam * weights (the transpose of one sample).
template <typename T>
__device__ __forceinline__ void stencil_scatter(T* __restrict__ lf, int64_t ld, const Stencil& s, double lam) {
  atomicAdd(lf + (int64_t)s.y0 * ld + s.x0, (T)(lam * (1.0 - s.tx) * (1.0 - s.ty)));
  atomicAdd(lf + (int64_t)s.y0 * ld + s.x1, (T)(lam * s.tx * (1.0 - s.ty)));
  atomicAdd(lf + (int64_t)s.y1 * ld + s.x0, (T)(lam * (1.0 - s.tx) * s.ty));
  atomicAdd(lf + (int64_t)s.y1 * ld + s.x1, (T)(lam * s.tx * s.ty));
}

// ------------------------------------------------------------------ control
// u[j, i] += dt fu[j, i] (i < W), v[j, i] += dt fv[j, i] (j < H): the control of step t acts
// on the left / lower face of each cell.
template <typename T>
__global__ void k_add_control(int H, int W, T* __restrict__ u, int64_t ldu, T* __restrict__ v, int64_t ldv,
                              const T* __restrict__ fu, int64_t ldfu, const T* __restrict__ fv, int64_t ldfv,
                              double dt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= W || j >= H) return;
  T* pu = u + (int64_t)j * ldu + i;
  T* pv = v + (int64_t)j * ldv + i;
  *pu = (T)((double)*pu + dt * (double)fu[(int64_t)j * ldfu + i]);
  *pv = (T)((double)*pv + dt * (double)fv[(int64_t)j * ldfv + i]);
}

// ------------------------------------------------------------------ density advection
// Per target cell: the transpose of the source sample (scatter, or a stored stencil for the
// gather) and lam_uu / lam_vv, the adjoints of the velocity sampled at the cell centre.
template <typename T>
__global__ void k_adj_advect_scalar(int H, int W, const T* __restrict__ lam_out, int64_t ldl,
                                    const T* __restrict__ src, int64_t lds, const T* __restrict__ u, int64_t ldu,
                                    const T* __restrict__ v, int64_t ldv, Masks m, double dt, double inv,
                                    double diss, T* __restrict__ lam_src, int64_t ldls, T* __restrict__ lam_uu,
                                    T* __restrict__ lam_vv, int4* __restrict__ sten_idx,
                                    double2* __restrict__ sten_w, int* __restrict__ radius) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= W || j >= H) return;
  const int64_t c = (int64_t)j * W + i;
  if (!m.fluid(j, i)) {
    lam_uu[c] = (T)0;
    lam_vv[c] = (T)0;
    if (sten_idx) sten_idx[c] = make_int4(-1, -1, -1, -1);
    return;
  }
  const double px = (double)i + 0.5, py = (double)j + 0.5;
  const Stencil su = stencil_ref(H, (int64_t)W + 1, px, py - 0.5);
  const Stencil sv = stencil_ref((int64_t)H + 1, W, px - 0.5, py);
  const double uu = stencil_value(u, ldu, su), vv = stencil_value(v, ldv, sv);
  const double x = px - uu * dt * inv, y = py - vv * dt * inv;
  const Stencil s = stencil_ref(H, W, x - 0.5, y - 0.5);
  const double lam = diss * (double)lam_out[(int64_t)j * ldl + i];
  if (sten_idx) {
    sten_idx[c] = make_int4(s.x0, s.x1, s.y0, s.y1);
    sten_w[c] = make_double2(s.tx, s.ty);
    const int r = max(max(abs(s.x0 - i), abs(s.x1 - i)), max(abs(s.y0 - j), abs(s.y1 - j)));
    atomicMax(radius, r);
  } else if (lam != 0.0) {
    stencil_scatter(lam_src, ldls, s, lam);
  }
  double gx, gy;
  stencil_grad(src, lds, s, gx, gy);
  lam_uu[c] = (T)(-lam * gx * dt * inv);
  lam_vv[c] = (T)(-lam * gy * dt * inv);
}

// Deterministic transpose: source cell (js, is) gathers diss * lam_out[t] * w(t -> s) over
// the targets t within the largest stencil reach, in a fixed order.
template <typename T>
__global__ void k_adj_gather_scalar(int H, int W, const T* __restrict__ lam_out, int64_t ldl,
                                    const int4* __restrict__ sten_idx, const double2* __restrict__ sten_w,
                                    const int* __restrict__ radius, double diss, T* __restrict__ lam_src,
                                    int64_t ldls) {
  const int is = blockIdx.x * blockDim.x + threadIdx.x;
  const int js = blockIdx.y * blockDim.y + threadIdx.y;
  if (is >= W || js >= H) return;
  const int R = *radius;
  double acc = 0.0;
  for (int dy = -R; dy <= R; ++dy) {
    const int j = js + dy;
    if (j < 0 || j >= H) continue;
    for (int dx = -R; dx <= R; ++dx) {
      const int i = is + dx;
      if (i < 0 || i >= W) continue;
      const int64_t c = (int64_t)j * W + i;
      const int4 q = sten_idx[c];
      if (q.x < 0) continue;
      const bool hx0 = q.x == is, hx1 = q.y == is, hy0 = q.z == js, hy1 = q.w == js;
      if (!(hx0 || hx1) || !(hy0 || hy1)) continue;
      const double2 t = sten_w[c];
      const double wx = (hx0 ? 1.0 - t.x : 0.0) + (hx1 ? t.x : 0.0);
      const double wy = (hy0 ? 1.0 - t.y : 0.0) + (hy1 ? t.y : 0.0);
      acc += wx * wy * (double)lam_out[(int64_t)j * ldl + i];
    }
  }
  T* p = lam_src + (int64_t)js * ldls + is;
  *p = (T)((double)*p + diss * acc);
}

// The centre velocity of target (j, i) is the mean of u[j, i], u[j, i + 1] (and of v[j, i],
// v[j + 1, i]): lam_u[j, i] += (lam_uu[j, i - 1] + lam_uu[j, i]) / 2 and likewise for v.
template <typename T>
__global__ void k_adj_centre_velocity(int H, int W, const T* __restrict__ lam_uu, const T* __restrict__ lam_vv,
                                      T* __restrict__ lam_u, int64_t ldu, T* __restrict__ lam_v, int64_t ldv) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (j < H && i <= W) {
    double a = 0.0;
    if (i < W) a += 0.5 * (double)lam_uu[(int64_t)j * W + i];
    if (i > 0) a += 0.5 * (double)lam_uu[(int64_t)j * W + i - 1];
    T* p = lam_u + (int64_t)j * ldu + i;
    *p = (T)((double)*p + a);
  }
  if (j <= H && i < W) {
    double a = 0.0;
    if (j < H) a += 0.5 * (double)lam_vv[(int64_t)j * W + i];
    if (j > 0) a += 0.5 * (double)lam_vv[(int64_t)(j - 1) * W + i];
    T* p = lam_v + (int64_t)j * ldv + i;
    *p = (T)((double)*p + a);
  }
}

// ------------------------------------------------------------------ velocity advection
// One thread per face of the MAC grid (grid covers (W + 1) x (H + 1)); scatters with atomics.
template <typename T>
__global__ void k_adj_advect_uv(int H, int W, const T* __restrict__ lam_un, int64_t ldlun,
                                const T* __restrict__ lam_vn, int64_t ldlvn, const T* __restrict__ u, int64_t ldu,
                                const T* __restrict__ v, int64_t ldv, Masks m, double dt, double inv,
                                T* __restrict__ lam_u, int64_t ldlu, T* __restrict__ lam_v, int64_t ldlv) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (j < H && i <= W && m.u(j, i)) {
    const double lam = (double)lam_un[(int64_t)j * ldlun + i];
    if (lam != 0.0) {
      // advection.py:130-154: u at the face itself, v sampled at (i - 0.5, j + 0.5)
      const double px = (double)i, py = (double)j + 0.5;
      const double uu = (double)u[(int64_t)j * ldu + i];
      const Stencil sv = stencil_ref((int64_t)H + 1, W, px - 0.5, py);
      const double vv = stencil_value(v, ldv, sv);
      const double x = px - uu * dt * inv, y = py - vv * dt * inv;
      const Stencil s = stencil_ref(H, (int64_t)W + 1, x, y - 0.5);
      stencil_scatter(lam_u, ldlu, s, lam);
      double gx, gy;
      stencil_grad(u, ldu, s, gx, gy);
      atomicAdd(lam_u + (int64_t)j * ldlu + i, (T)(-lam * gx * dt * inv));
      stencil_scatter(lam_v, ldlv, sv, -lam * gy * dt * inv);
    }
  }
  if (j <= H && i < W && m.v(j, i)) {
    const double lam = (double)lam_vn[(int64_t)j * ldlvn + i];
    if (lam != 0.0) {
      // advection.py:156-180: u sampled at (i + 0.5, j - 0.5), v at the face itself
      const double px = (double)i + 0.5, py = (double)j;
      const Stencil su = stencil_ref(H, (int64_t)W + 1, px, py - 0.5);
      const double uu = stencil_value(u, ldu, su);
      const double vv = (double)v[(int64_t)j * ldv + i];
      const double x = px - uu * dt * inv, y = py - vv * dt * inv;
      const Stencil s = stencil_ref((int64_t)H + 1, W, x - 0.5, y);
      stencil_scatter(lam_v, ldlv, s, lam);
      double gx, gy;
      stencil_grad(v, ldv, s, gx, gy);
      atomicAdd(lam_v + (int64_t)j * ldlv + i, (T)(-lam * gy * dt * inv));
      stencil_scatter(lam_u, ldlu, su, -lam * gx * dt * inv);
    }
  }
}

// ------------------------------------------------------------------ forces and control
// forces.py:19-46 as a linear map of density onto v faces: face j takes d[j] alone at j = 0
// and j = H - 1, (d[j - 1] + d[j]) / 2 between, nothing at j = H; scaled by -dc g dt.
// lam_d[j, i] += dt (-dc g) (cs(j) lam_v[j, i] + cp(j + 1) lam_v[j + 1, i]); the control
// gradients are dt lam_u[j, i] (i < W) and dt lam_v[j, i] (j < H).
template <typename T>
__global__ void k_adj_forces(int H, int W, const T* __restrict__ lam_u, int64_t ldlu, const T* __restrict__ lam_v,
                             int64_t ldlv, T* __restrict__ lam_d, int64_t ldld, T* __restrict__ gfu, int64_t ldgu,
                             T* __restrict__ gfv, int64_t ldgv, double dt, double g, double dc) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= W || j >= H) return;
  const double k = -dc * g * dt;
  const double cs = (j == 0 || j == H - 1) ? 1.0 : 0.5;
  const int jn = j + 1;
  const double cp = (jn >= 1 && jn <= H - 2) ? 0.5 : 0.0;
  const double lv = (double)lam_v[(int64_t)j * ldlv + i];
  double a = cs * lv;
  if (cp != 0.0) a += cp * (double)lam_v[(int64_t)jn * ldlv + i];
  T* pd = lam_d + (int64_t)j * ldld + i;
  *pd = (T)((double)*pd + k * a);
  if (gfu) gfu[(int64_t)j * ldgu + i] = (T)(dt * (double)lam_u[(int64_t)j * ldlu + i]);
  if (gfv) gfv[(int64_t)j * ldgv + i] = (T)(dt * lv);
}

// ------------------------------------------------------------------ projection
// pressure_gradient.py:4-37 + boundaries.py:7-39: u''[f] = o(f) (u'[f] - s (p_right - p_left))
// with o(f) = 1 on open faces not next to a solid cell. lam_u' = o lam_u'' and
// lam_p = -s G^T (o lam_u''), G the face difference of the cell pressures.
__device__ __forceinline__ bool open_u(const Masks& m, int solid_mode, const uint8_t* solid, int64_t lds, int H, int W,
                                       int j, int i) {
  if (i <= 0 || i >= W || !m.u(j, i)) return false;
  return !(solid_at(solid_mode, solid, lds, H, W, j, i - 1) || solid_at(solid_mode, solid, lds, H, W, j, i));
}

__device__ __forceinline__ bool open_v(const Masks& m, int solid_mode, const uint8_t* solid, int64_t lds, int H, int W,
                                       int j, int i) {
  if (j <= 0 || j >= H || !m.v(j, i)) return false;
  return !(solid_at(solid_mode, solid, lds, H, W, j - 1, i) || solid_at(solid_mode, solid, lds, H, W, j, i));
}

template <typename T>
__global__ void k_adj_project(int H, int W, const T* __restrict__ lu, int64_t ldlu, const T* __restrict__ lv,
                              int64_t ldlv, T* __restrict__ lu_out, int64_t ldou, T* __restrict__ lv_out, int64_t ldov,
                              T* __restrict__ lam_p, int64_t ldp, Masks m, int solid_mode,
                              const uint8_t* __restrict__ solid, int64_t lds, double scale) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (j < H && i <= W)
    lu_out[(int64_t)j * ldou + i] =
        open_u(m, solid_mode, solid, lds, H, W, j, i) ? lu[(int64_t)j * ldlu + i] : (T)0;
  if (j <= H && i < W)
    lv_out[(int64_t)j * ldov + i] =
        open_v(m, solid_mode, solid, lds, H, W, j, i) ? lv[(int64_t)j * ldlv + i] : (T)0;
  if (j < H && i < W) {
    double a = 0.0;
    if (open_u(m, solid_mode, solid, lds, H, W, j, i)) a += (double)lu[(int64_t)j * ldlu + i];
    if (open_u(m, solid_mode, solid, lds, H, W, j, i + 1)) a -= (double)lu[(int64_t)j * ldlu + i + 1];
    if (open_v(m, solid_mode, solid, lds, H, W, j, i)) a += (double)lv[(int64_t)j * ldlv + i];
    if (open_v(m, solid_mode, solid, lds, H, W, j + 1, i)) a -= (double)lv[(int64_t)(j + 1) * ldlv + i];
    lam_p[(int64_t)j * ldp + i] = (T)(-scale * a);
  }
}

// divergence.py:4-25 transposed: face u[j, i] enters div[j, i - 1] with + and div[j, i] with
// -, each times its mask and 1 / h.
template <typename T>
__global__ void k_adj_divergence(int H, int W, const T* __restrict__ ldiv, int64_t ldd, T* __restrict__ lu,
                                 int64_t ldlu, T* __restrict__ lv, int64_t ldlv, Masks m, double inv) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (j < H && i <= W && m.u(j, i)) {
    double a = 0.0;
    if (i >= 1) a += (double)ldiv[(int64_t)j * ldd + i - 1];
    if (i < W) a -= (double)ldiv[(int64_t)j * ldd + i];
    T* p = lu + (int64_t)j * ldlu + i;
    *p = (T)((double)*p + inv * a);
  }
  if (j <= H && i < W && m.v(j, i)) {
    double a = 0.0;
    if (j >= 1) a += (double)ldiv[(int64_t)(j - 1) * ldd + i];
    if (j < H) a -= (double)ldiv[(int64_t)j * ldd + i];
    T* p = lv + (int64_t)j * ldlv + i;
    *p = (T)((double)*p + inv * a);
  }
}

static int grid_ok(int64_t H, int64_t W) {
  if (H < 1 || W < 1 || H > (1 << 16) || W > (1 << 16)) return fail(SG_ERR_ARG, "bad grid %lld x %lld", (long long)H,
                                                                    (long long)W);
  return SG_OK;
}

static int masks_of(int mode, int64_t H, int64_t W, const uint8_t* fmu, int64_t ldu, const uint8_t* fmv, int64_t ldv,
                    const uint8_t* fl, int64_t ldf, Masks& m) {
  if (mode != SG_MASK_PLANES && mode != SG_MASK_OPEN && mode != SG_MASK_RING) return fail(SG_ERR_ARG, "bad mask mode");
  if (mode == SG_MASK_PLANES && !((fmu && fmv) || fl)) return fail(SG_ERR_ARG, "mask planes required");
  m = make_masks(mode, H, W, fmu, ldu, fmv, ldv, fl, ldf);
  return SG_OK;
}

}  // namespace sg

using namespace sg;

extern "C" {

int sg_add_control(int dtype, int64_t H, int64_t W, void* u, int64_t ld_u, void* v, int64_t ld_v, const void* fu,
                   int64_t ld_fu, const void* fv, int64_t ld_fv, double dt, void* stream) {
  SG_CHECK(grid_ok(H, W));
  SG_REQUIRE(u && v && fu && fv, "null field pointer");
  SG_REQUIRE(ld_u >= W + 1 && ld_v >= W && ld_fu >= W && ld_fv >= W, "row stride below row length");
  SG_DISPATCH(dtype, {
    SG_LAUNCH(k_add_control<T><<<grid2d(W, H), block2d(), 0, as_stream(stream)>>>(
        (int)H, (int)W, (T*)u, ld_u, (T*)v, ld_v, (const T*)fu, ld_fu, (const T*)fv, ld_fv, dt));
  });
  return check_launch("sg_add_control");
}

int64_t sg_adjoint_advect_scalar_workspace(int dtype, int64_t H, int64_t W, int gather) {
  const int64_t n = H * W, es = dtype == SG_F64 ? 8 : 4;
  int64_t bytes = ((2 * n * es + 255) / 256) * 256;
  if (gather) bytes += n * (int64_t)(sizeof(int4) + sizeof(double2)) + 256;
  return bytes;
}

int sg_adjoint_advect_scalar(int dtype, int64_t H, int64_t W, const void* lam_out, int64_t ld_lo, const void* src,
                             int64_t ld_src, const void* u, int64_t ld_u, const void* v, int64_t ld_v, int mask_mode,
                             const uint8_t* is_fluid, int64_t ld_fluid, double dt, double cell_size,
                             double dissipation, void* lam_src, int64_t ld_ls, void* lam_u, int64_t ld_lu, void* lam_v,
                             int64_t ld_lv, int gather, void* workspace, int64_t workspace_bytes, void* stream) {
  SG_CHECK(grid_ok(H, W));
  SG_REQUIRE(lam_out && src && u && v && lam_src && lam_u && lam_v && workspace, "null pointer");
  SG_REQUIRE(ld_lo >= W && ld_src >= W && ld_u >= W + 1 && ld_v >= W && ld_ls >= W && ld_lu >= W + 1 && ld_lv >= W,
             "row stride below row length");
  SG_REQUIRE(cell_size > 0.0, "cell_size must be positive");
  SG_REQUIRE(workspace_bytes >= sg_adjoint_advect_scalar_workspace(dtype, H, W, gather),
             "workspace below sg_adjoint_advect_scalar_workspace()");
  Masks m;
  SG_CHECK(masks_of(mask_mode, H, W, nullptr, 0, nullptr, 0, is_fluid, ld_fluid, m));
  cudaStream_t s = as_stream(stream);
  const int64_t n = H * W;
  SG_DISPATCH(dtype, {
    T* luu = (T*)workspace;
    T* lvv = luu + n;
    char* tail = (char*)workspace + ((2 * n * (int64_t)sizeof(T) + 255) / 256) * 256;
    int4* sidx = gather ? (int4*)tail : nullptr;
    double2* sw = gather ? (double2*)(tail + n * (int64_t)sizeof(int4)) : nullptr;
    int* radius = gather ? (int*)(tail + n * (int64_t)(sizeof(int4) + sizeof(double2))) : nullptr;
    if (gather) {
      cudaError_t e = cudaMemsetAsync(radius, 0, sizeof(int), s);
      if (e != cudaSuccess) return fail(SG_ERR_CUDA, "memset: %s", cudaGetErrorString(e));
    }
    SG_LAUNCH(k_adj_advect_scalar<T><<<grid2d(W, H), block2d(), 0, s>>>(
        (int)H, (int)W, (const T*)lam_out, ld_lo, (const T*)src, ld_src, (const T*)u, ld_u, (const T*)v, ld_v, m, dt,
        1.0 / cell_size, dissipation, (T*)lam_src, ld_ls, luu, lvv, sidx, sw, radius));
    if (gather)
      SG_LAUNCH(k_adj_gather_scalar<T><<<grid2d(W, H), block2d(), 0, s>>>(
          (int)H, (int)W, (const T*)lam_out, ld_lo, sidx, sw, radius, dissipation, (T*)lam_src, ld_ls));
    SG_LAUNCH(k_adj_centre_velocity<T><<<grid2d(W + 1, H + 1), block2d(), 0, s>>>((int)H, (int)W, luu, lvv,
                                                                                  (T*)lam_u, ld_lu, (T*)lam_v, ld_lv));
  });
  return check_launch("sg_adjoint_advect_scalar");
}

int sg_adjoint_advect_velocity(int dtype, int64_t H, int64_t W, const void* lam_u_new, int64_t ld_lun,
                               const void* lam_v_new, int64_t ld_lvn, const void* u, int64_t ld_u, const void* v,
                               int64_t ld_v, int mask_mode, const uint8_t* fmu, int64_t ld_fmu, const uint8_t* fmv,
                               int64_t ld_fmv, double dt, double cell_size, void* lam_u, int64_t ld_lu, void* lam_v,
                               int64_t ld_lv, void* stream) {
  SG_CHECK(grid_ok(H, W));
  SG_REQUIRE(lam_u_new && lam_v_new && u && v && lam_u && lam_v, "null pointer");
  SG_REQUIRE(ld_lun >= W + 1 && ld_lvn >= W && ld_u >= W + 1 && ld_v >= W && ld_lu >= W + 1 && ld_lv >= W,
             "row stride below row length");
  SG_REQUIRE(cell_size > 0.0, "cell_size must be positive");
  Masks m;
  SG_CHECK(masks_of(mask_mode, H, W, fmu, ld_fmu, fmv, ld_fmv, nullptr, 0, m));
  SG_DISPATCH(dtype, {
    SG_LAUNCH(k_adj_advect_uv<T><<<grid2d(W + 1, H + 1), block2d(), 0, as_stream(stream)>>>(
        (int)H, (int)W, (const T*)lam_u_new, ld_lun, (const T*)lam_v_new, ld_lvn, (const T*)u, ld_u, (const T*)v, ld_v,
        m, dt, 1.0 / cell_size, (T*)lam_u, ld_lu, (T*)lam_v, ld_lv));
  });
  return check_launch("sg_adjoint_advect_velocity");
}

int sg_adjoint_forces(int dtype, int64_t H, int64_t W, const void* lam_u, int64_t ld_lu, const void* lam_v,
                      int64_t ld_lv, void* lam_d, int64_t ld_ld, void* grad_fu, int64_t ld_gu, void* grad_fv,
                      int64_t ld_gv, double dt, double gravity, double density_coefficient, void* stream) {
  SG_CHECK(grid_ok(H, W));
  SG_REQUIRE(lam_u && lam_v && lam_d, "null pointer");
  SG_REQUIRE(ld_lu >= W + 1 && ld_lv >= W && ld_ld >= W && (!grad_fu || ld_gu >= W) && (!grad_fv || ld_gv >= W),
             "row stride below row length");
  SG_DISPATCH(dtype, {
    SG_LAUNCH(k_adj_forces<T><<<grid2d(W, H), block2d(), 0, as_stream(stream)>>>(
        (int)H, (int)W, (const T*)lam_u, ld_lu, (const T*)lam_v, ld_lv, (T*)lam_d, ld_ld, (T*)grad_fu, ld_gu,
        (T*)grad_fv, ld_gv, dt, gravity, density_coefficient));
  });
  return check_launch("sg_adjoint_forces");
}

int sg_adjoint_project(int dtype, int64_t H, int64_t W, const void* lam_u, int64_t ld_lu, const void* lam_v,
                       int64_t ld_lv, void* lam_u_out, int64_t ld_lou, void* lam_v_out, int64_t ld_lov, void* lam_p,
                       int64_t ld_lp, int mask_mode, const uint8_t* fmu, int64_t ld_fmu, const uint8_t* fmv,
                       int64_t ld_fmv, int solid_mode, const uint8_t* solid, int64_t ld_s, double fluid_density,
                       double cell_size, double dt, void* stream) {
  SG_CHECK(grid_ok(H, W));
  SG_REQUIRE(lam_u && lam_v && lam_u_out && lam_v_out && lam_p, "null pointer");
  SG_REQUIRE(ld_lu >= W + 1 && ld_lv >= W && ld_lou >= W + 1 && ld_lov >= W && ld_lp >= W,
             "row stride below row length");
  SG_REQUIRE(solid_mode != SG_MASK_PLANES || solid, "solid plane required");
  SG_REQUIRE(fluid_density > 0.0 && cell_size > 0.0, "density and cell size must be positive");
  Masks m;
  SG_CHECK(masks_of(mask_mode, H, W, fmu, ld_fmu, fmv, ld_fmv, nullptr, 0, m));
  const double scale = dt / (fluid_density * cell_size);
  SG_DISPATCH(dtype, {
    SG_LAUNCH(k_adj_project<T><<<grid2d(W + 1, H + 1), block2d(), 0, as_stream(stream)>>>(
        (int)H, (int)W, (const T*)lam_u, ld_lu, (const T*)lam_v, ld_lv, (T*)lam_u_out, ld_lou, (T*)lam_v_out, ld_lov,
        (T*)lam_p, ld_lp, m, solid_mode, solid, ld_s, scale));
  });
  return check_launch("sg_adjoint_project");
}

int sg_adjoint_divergence(int dtype, int64_t H, int64_t W, const void* lam_div, int64_t ld_ld, void* lam_u,
                          int64_t ld_lu, void* lam_v, int64_t ld_lv, int mask_mode, const uint8_t* fmu, int64_t ld_fmu,
                          const uint8_t* fmv, int64_t ld_fmv, double cell_size, void* stream) {
  SG_CHECK(grid_ok(H, W));
  SG_REQUIRE(lam_div && lam_u && lam_v, "null pointer");
  SG_REQUIRE(ld_ld >= W && ld_lu >= W + 1 && ld_lv >= W, "row stride below row length");
  SG_REQUIRE(cell_size > 0.0, "cell_size must be positive");
  Masks m;
  SG_CHECK(masks_of(mask_mode, H, W, fmu, ld_fmu, fmv, ld_fmv, nullptr, 0, m));
  SG_DISPATCH(dtype, {
    SG_LAUNCH(k_adj_divergence<T><<<grid2d(W + 1, H + 1), block2d(), 0, as_stream(stream)>>>(
        (int)H, (int)W, (const T*)lam_div, ld_ld, (T*)lam_u, ld_lu, (T*)lam_v, ld_lv, m, 1.0 / cell_size));
  });
  return check_launch("sg_adjoint_divergence");
}

}  // extern "C"

SG_BOUNDS_ACCESSOR(adjoint)
