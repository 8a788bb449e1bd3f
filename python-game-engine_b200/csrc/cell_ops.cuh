// Per-cell bodies of the smoke-step operators, shared by the single-grid kernels
// (operators.cu) and the batched ones (batch.cu) so both compute every cell the same way.
// Both units are compiled with -fmad=false (no FMA contraction): the arithmetic rounds as
// the reference's Numba kernels do.
#pragma once

#include "common.cuh"

namespace sg {

// advection.py:112-128 (+ dissipation, simulation.py:232): the new value of cell (j, i).
template <typename T, typename MK>
__device__ __forceinline__ T advect_scalar_cell(int j, int i, int H, int W, const T* __restrict__ src, int64_t lds,
                                                const T* __restrict__ u, int64_t ur, int64_t uc, int64_t ldu,
                                                const T* __restrict__ v, int64_t vr, int64_t vc, int64_t ldv,
                                                const MK& m, double dt, double inv, T diss) {
  if (!m.fluid(j, i)) return (T)0;
  double px = idx_double(i) + 0.5, py = idx_double(j) + 0.5;
  double uu = sample_ref(u, ldu, ur, uc, px, py - 0.5);
  double vv = sample_ref(v, ldv, vr, vc, px - 0.5, py);
  double x = px - (uu * dt * inv);
  double y = py - (vv * dt * inv);
  T val = (T)sample_ref(src, lds, (int64_t)H, (int64_t)W, x - 0.5, y - 0.5);
  return val * diss;
}

// advection.py:130-154
template <typename T>
__device__ __forceinline__ T advect_u_face(int j, int i, const T* __restrict__ us, int64_t ldus, int64_t ur, int64_t uc,
                                           const T* __restrict__ v, int64_t vr, int64_t vc, int64_t ldv, double dt,
                                           double inv) {
  double px = idx_double(i), py = idx_double(j) + 0.5;
  T uu = us[(int64_t)j * ldus + i];
  double vv = sample_ref(v, ldv, vr, vc, px - 0.5, py);
  double x = px - ((double)uu * dt * inv);
  double y = py - (vv * dt * inv);
  return (T)sample_ref(us, ldus, ur, uc, x, y - 0.5);
}

// advection.py:156-180
template <typename T>
__device__ __forceinline__ T advect_v_face(int j, int i, const T* __restrict__ vs, int64_t ldvs, int64_t vr, int64_t vc,
                                           const T* __restrict__ u, int64_t ur, int64_t uc, int64_t ldu, double dt,
                                           double inv) {
  double px = idx_double(i) + 0.5, py = idx_double(j);
  double uu = sample_ref(u, ldu, ur, uc, px, py - 0.5);
  T vv = vs[(int64_t)j * ldvs + i];
  double x = px - (uu * dt * inv);
  double y = py - ((double)vv * dt * inv);
  return (T)sample_ref(vs, ldvs, vr, vc, x - 0.5, y);
}

// forces.py:19-105. v is (H+1) x W.
template <typename T>
__device__ __forceinline__ void forces_face(int j, int i, int H, int W, T* __restrict__ v, int64_t ldv,
                                            const T* __restrict__ d, int64_t ldd, const T* __restrict__ t, int64_t ldt,
                                            double dt, double g, double bc, double dc, double amb, int f32tmp) {
  double bf = 0.0;
  if (j < H) {
    double dd;
    if (j == 0 || j == H - 1) {
      dd = (double)d[(int64_t)j * ldd + i];
    } else {
      T s = d[(int64_t)(j - 1) * ldd + i] + d[(int64_t)j * ldd + i];
      dd = 0.5 * (double)s;
    }
    bf = -dc * dd * g;
  }
  double tt;
  if (t == nullptr) {
    tt = amb;
  } else if (j == 0) {
    tt = (double)t[i];
  } else if (j == H) {
    tt = (double)t[(int64_t)(H - 1) * ldt + i];
  } else {
    T s = t[(int64_t)(j - 1) * ldt + i] + t[(int64_t)j * ldt + i];
    tt = 0.5 * (double)s;
  }
  double tf = -bc * (tt - amb);
  double add;
  if (f32tmp) {
    float b32 = (float)bf, t32 = (float)tf;
    float s = b32 + t32;
    add = dt * (double)s;
  } else {
    add = dt * (bf + tf);
  }
  int64_t k = (int64_t)j * ldv + i;
  v[k] = (T)((double)v[k] + add);
}

// divergence.py:4-25: divergence of cell (j, i).
template <typename T, typename MK>
__device__ __forceinline__ T divergence_cell(int j, int i, const T* __restrict__ u, int64_t ldu, const T* __restrict__ v,
                                             int64_t ldv, const MK& m, double inv) {
  T a = u[(int64_t)j * ldu + i + 1] * (T)(m.u(j, i + 1) ? 1 : 0);
  T b = u[(int64_t)j * ldu + i] * (T)(m.u(j, i) ? 1 : 0);
  T c = v[(int64_t)(j + 1) * ldv + i] * (T)(m.v(j + 1, i) ? 1 : 0);
  T e = v[(int64_t)j * ldv + i] * (T)(m.v(j, i) ? 1 : 0);
  T du = a - b, dv = c - e;
  return (T)((double)du * inv + (double)dv * inv);
}

// Masked neighbour sum shared with jacobi.py:18-21 and red_black_sor_gauss_seidel.py:19-22.
template <typename T, typename MK>
__device__ __forceinline__ T nbsum_ref(const T* __restrict__ p, int64_t ld, int H, int W, int j, int i, const MK& m,
                                       T c) {
  T l = m.u(j, i) ? p[(int64_t)j * ld + (i - 1 > 0 ? i - 1 : 0)] : c;
  T r = m.u(j, i + 1) ? p[(int64_t)j * ld + (i + 1 < W - 1 ? i + 1 : W - 1)] : c;
  T d = m.v(j, i) ? p[(int64_t)(j - 1 > 0 ? j - 1 : 0) * ld + i] : c;
  T up = m.v(j + 1, i) ? p[(int64_t)(j + 1 < H - 1 ? j + 1 : H - 1) * ld + i] : c;
  T s = l + r;
  s = s + d;
  s = s + up;
  return s;
}

// residual.py:6-42: the residual of cell (j, i) (0 off the fluid).
template <typename T, typename MK>
__device__ __forceinline__ T residual_cell(int j, int i, int H, int W, const T* __restrict__ p, int64_t ldp,
                                           const T* __restrict__ div, int64_t ldd, const MK& m, double alpha,
                                           double beta) {
  if (!m.fluid(j, i)) return (T)0;
  T c = p[(int64_t)j * ldp + i];
  T s = nbsum_ref(p, ldp, H, W, j, i, m, c);
  return (T)(((double)s + alpha * (double)div[(int64_t)j * ldd + i]) - beta * (double)c);
}

// pressure_gradient.py:4-37 then, if solid_mode != SG_MASK_NONE, boundaries.py:7-39: the
// projected value of u face (j, i) (j < H, i <= W) from the face's current value uk.
template <typename T, typename MK, int SM = -1>
__device__ __forceinline__ T projected_u(int j, int i, int H, int W, T uk, const T* __restrict__ p, int64_t ldp,
                                         const MK& m, int do_grad, int solid_mode,
                                         const uint8_t* __restrict__ solid, int64_t lds, double scale) {
  bool zero = (i > 0 && solid_at_t<SM>(solid_mode, solid, lds, H, W, j, i - 1)) ||
              (i < W && solid_at_t<SM>(solid_mode, solid, lds, H, W, j, i));
  if (zero) return (T)0;
  if (!do_grad) return uk;
  if (m.u(j, i) && i > 0 && i < W) {
    T dp = p[(int64_t)j * ldp + i] - p[(int64_t)j * ldp + i - 1];
    return (T)((double)uk - scale * (double)dp);
  }
  return (T)0;
}

// the same for v face (j, i) (j <= H, i < W)
template <typename T, typename MK, int SM = -1>
__device__ __forceinline__ T projected_v(int j, int i, int H, int W, T vk, const T* __restrict__ p, int64_t ldp,
                                         const MK& m, int do_grad, int solid_mode,
                                         const uint8_t* __restrict__ solid, int64_t lds, double scale) {
  bool zero = (j > 0 && solid_at_t<SM>(solid_mode, solid, lds, H, W, j - 1, i)) ||
              (j < H && solid_at_t<SM>(solid_mode, solid, lds, H, W, j, i));
  if (zero) return (T)0;
  if (!do_grad) return vk;
  if (m.v(j, i) && j > 0 && j < H) {
    T dp = p[(int64_t)j * ldp + i] - p[(int64_t)(j - 1) * ldp + i];
    return (T)((double)vk - scale * (double)dp);
  }
  return (T)0;
}

// Projection of u face (j, i) (j < H, i <= W) and v face (j, i) (j <= H, i < W) in place.
template <typename T, typename MK, int SM = -1>
__device__ __forceinline__ void project_faces(int j, int i, int H, int W, T* __restrict__ u, int64_t ldu,
                                              T* __restrict__ v, int64_t ldv, const T* __restrict__ p, int64_t ldp,
                                              const MK& m, int do_grad, int solid_mode,
                                              const uint8_t* __restrict__ solid, int64_t lds, double scale) {
  if (j < H && i <= W) {
    T* q = u + (int64_t)j * ldu + i;
    *q = projected_u<T, MK, SM>(j, i, H, W, *q, p, ldp, m, do_grad, solid_mode, solid, lds, scale);
  }
  if (j <= H && i < W) {
    T* q = v + (int64_t)j * ldv + i;
    *q = projected_v<T, MK, SM>(j, i, H, W, *q, p, ldp, m, do_grad, solid_mode, solid, lds, scale);
  }
}

// projected_u / projected_v (gradient branch) from the pressure values at the face's two
// cells, pc = p(j, i) and pn = p(j, i - 1) (u) or p(j - 1, i) (v), with the same
// expressions; the values are read only where the reference reads them.
template <typename T, typename MK, int SM>
__device__ __forceinline__ T projected_u_pv(int j, int i, int H, int W, T uk, T pc, T pn, const MK& m, int solid_mode,
                                           const uint8_t* __restrict__ solid, int64_t lds, double scale) {
  bool zero = (i > 0 && solid_at_t<SM>(solid_mode, solid, lds, H, W, j, i - 1)) ||
              (i < W && solid_at_t<SM>(solid_mode, solid, lds, H, W, j, i));
  if (zero) return (T)0;
  if (m.u(j, i) && i > 0 && i < W) {
    T dp = pc - pn;
    return (T)((double)uk - scale * (double)dp);
  }
  return (T)0;
}

template <typename T, typename MK, int SM>
__device__ __forceinline__ T projected_v_pv(int j, int i, int H, int W, T vk, T pc, T pn, const MK& m, int solid_mode,
                                           const uint8_t* __restrict__ solid, int64_t lds, double scale) {
  bool zero = (j > 0 && solid_at_t<SM>(solid_mode, solid, lds, H, W, j - 1, i)) ||
              (j < H && solid_at_t<SM>(solid_mode, solid, lds, H, W, j, i));
  if (zero) return (T)0;
  if (m.v(j, i) && j > 0 && j < H) {
    T dp = pc - pn;
    return (T)((double)vk - scale * (double)dp);
  }
  return (T)0;
}

// divergence.py:4-25 of cell (j, i) from its four face values (ul, ur: u faces i, i + 1;
// vd, vu: v faces j, j + 1).
template <typename T, typename MK>
__device__ __forceinline__ T divergence_from_faces(int j, int i, T ul, T ur, T vd, T vu, const MK& m, double inv) {
  T a = ur * (T)(m.u(j, i + 1) ? 1 : 0);
  T b = ul * (T)(m.u(j, i) ? 1 : 0);
  T c = vu * (T)(m.v(j + 1, i) ? 1 : 0);
  T e = vd * (T)(m.v(j, i) ? 1 : 0);
  T du = a - b, dv = c - e;
  return (T)((double)du * inv + (double)dv * inv);
}

// residual.py:6-42 of cell (j, i) from the pressure values around it (pl, pr, pd, pu: the
// neighbours at i - 1, i + 1, j - 1, j + 1, read only inside the grid) and its divergence.
template <typename T, typename MK>
__device__ __forceinline__ T residual_from_values(int j, int i, int H, int W, T c, T pl, T pr, T pd, T pu, T dval,
                                                  const MK& m, double alpha, double beta) {
  if (!m.fluid(j, i)) return (T)0;
  T l = m.u(j, i) ? (i > 0 ? pl : c) : c;  // p[j, max(i - 1, 0)]
  T r = m.u(j, i + 1) ? (i < W - 1 ? pr : c) : c;
  T d = m.v(j, i) ? (j > 0 ? pd : c) : c;
  T up = m.v(j + 1, i) ? (j < H - 1 ? pu : c) : c;
  T s = l + r;
  s = s + d;
  s = s + up;
  return (T)(((double)s + alpha * (double)dval) - beta * (double)c);
}

// Overwriting disc sources at cell (j, i), u face (j, i) and v face (j, i) (j <= H, i <= W):
// the last of the n rows (cx, cy, r, density, v, noise) containing a point wins.
template <typename T>
__device__ __forceinline__ void plume_point(int j, int i, int H, int W, T* __restrict__ d, int64_t ldd,
                                            T* __restrict__ u, int64_t ldu, T* __restrict__ v, int64_t ldv,
                                            const double* src, int n, uint64_t seed, int64_t step) {
  int hit_d = -1, hit_v = -1, hit_u = -1;
  for (int s = 0; s < n; ++s) {
    double cx = src[6 * s], cy = src[6 * s + 1], r = src[6 * s + 2];
    double r2 = r * r;
    double dx = (double)i + 0.5 - cx, dy = (double)j + 0.5 - cy;
    if (j < H && i < W && dx * dx + dy * dy < r2) hit_d = s;
    dy = (double)j - cy;
    if (i < W && dx * dx + dy * dy < r2) hit_v = s;
    dx = (double)i - cx;
    dy = (double)j + 0.5 - cy;
    if (j < H && dx * dx + dy * dy < r2) hit_u = s;
  }
  if (hit_d >= 0) d[(int64_t)j * ldd + i] = (T)src[6 * hit_d + 3];
  if (hit_v >= 0)
    v[(int64_t)j * ldv + i] = (T)(src[6 * hit_v + 4] + noise(seed, step, 1, j, i, src[6 * hit_v + 5]));
  if (hit_u >= 0) u[(int64_t)j * ldu + i] = (T)noise(seed, step, 0, j, i, src[6 * hit_u + 5]);
}

}  // namespace sg
