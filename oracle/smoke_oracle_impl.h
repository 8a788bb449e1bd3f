/*
 * CPU oracle kernels, instantiated twice by smoke_oracle.c (REAL = float with
 * suffix _f32, REAL = double with suffix _f64).
 *
 * TEST INFRASTRUCTURE ONLY: this code is the checker for the CUDA path and the
 * CPU baseline that bench.py times beside it. Nothing in the product imports it.
 *
 * Each function restates one Numba kernel of the reference (LCEBurton/python-game-engine,
 * src/cfd/...) and mirrors Numba's arithmetic types: a float32 element combined with
 * a float32 element stays float32, anything combined with a Python float
 * (float64) is promoted to float64, and the final store rounds to REAL.
 * Arrays are row-major and contiguous; masks are one byte per entry (0/1).
 */

#define CAT2(a, b) a##b
#define CAT(a, b) CAT2(a, b)
#define FN(name) CAT(name, SFX)

static inline long FN(clampl)(long v, long lo, long hi) {
  /* backends/numba/operators/advection.py:6-14 (clamp) */
  if (v < lo) return lo;
  if (v > hi) return hi;
  return v;
}

static inline double FN(lerp_rr)(REAL a, REAL b, double t) {
  /* advection.py:16-19 with REAL endpoints: (b - a) is evaluated in REAL. */
  REAL d = b - a;
  return (double)a + (double)d * t;
}

/* backends/numba/operators/advection.py:21-49 (sample_scalar_field) */
static inline double FN(sample)(const REAL* f, long H, long W, double x, double y) {
  long x0 = (long)floor(x), x1 = (long)ceil(x);
  long y0 = (long)floor(y), y1 = (long)ceil(y);
  x0 = FN(clampl)(x0, 0, W - 1);
  x1 = FN(clampl)(x1, 0, W - 1);
  y0 = FN(clampl)(y0, 0, H - 1);
  y1 = FN(clampl)(y1, 0, H - 1);
  double tx = x - (double)x0;
  double ty = y - (double)y0;
  REAL c00 = f[y0 * W + x0], c10 = f[y0 * W + x1];
  REAL c01 = f[y1 * W + x0], c11 = f[y1 * W + x1];
  double c0 = FN(lerp_rr)(c00, c10, tx);
  double c1 = FN(lerp_rr)(c01, c11, tx);
  return c0 + (c1 - c0) * ty;
}

/* advection.py:112-128 (advect_scalar_field). u is (uH,uW), v is (vH,vW). */
void FN(or_advect_scalar)(const REAL* src, REAL* dst, long H, long W,
                          const REAL* u, long uH, long uW, const REAL* v, long vH, long vW,
                          const unsigned char* is_fluid, double dt, double h) {
  double inv = 1.0 / h;
#pragma omp parallel for schedule(static)
  for (long j = 0; j < H; ++j) {
    for (long i = 0; i < W; ++i) {
      if (!is_fluid[j * W + i]) { dst[j * W + i] = (REAL)0; continue; }
      double px = (double)i + 0.5, py = (double)j + 0.5;
      double uu = FN(sample)(u, uH, uW, px, py - 0.5);
      double vv = FN(sample)(v, vH, vW, px - 0.5, py);
      double x = px - (uu * dt * inv);
      double y = py - (vv * dt * inv);
      dst[j * W + i] = (REAL)FN(sample)(src, H, W, x - 0.5, y - 0.5);
    }
  }
}

/* advection.py:130-154 (advect_velocity_u) */
void FN(or_advect_u)(const REAL* usrc, REAL* udst, long uH, long uW,
                     const REAL* v, long vH, long vW, const unsigned char* fmu,
                     double dt, double h) {
  double inv = 1.0 / h;
#pragma omp parallel for schedule(static)
  for (long j = 0; j < uH; ++j) {
    for (long i = 0; i < uW; ++i) {
      if (!fmu[j * uW + i]) { udst[j * uW + i] = (REAL)0; continue; }
      double px = (double)i, py = (double)j + 0.5;
      REAL uu = usrc[j * uW + i];
      double vv = FN(sample)(v, vH, vW, px - 0.5, py);
      double x = px - ((double)uu * dt * inv);
      double y = py - (vv * dt * inv);
      udst[j * uW + i] = (REAL)FN(sample)(usrc, uH, uW, x, y - 0.5);
    }
  }
}

/* advection.py:156-180 (advect_velocity_v) */
void FN(or_advect_v)(const REAL* vsrc, REAL* vdst, long vH, long vW,
                     const REAL* u, long uH, long uW, const unsigned char* fmv,
                     double dt, double h) {
  double inv = 1.0 / h;
#pragma omp parallel for schedule(static)
  for (long j = 0; j < vH; ++j) {
    for (long i = 0; i < vW; ++i) {
      if (!fmv[j * vW + i]) { vdst[j * vW + i] = (REAL)0; continue; }
      double px = (double)i + 0.5, py = (double)j;
      double uu = FN(sample)(u, uH, uW, px, py - 0.5);
      REAL vv = vsrc[j * vW + i];
      double x = px - (uu * dt * inv);
      double y = py - ((double)vv * dt * inv);
      vdst[j * vW + i] = (REAL)FN(sample)(vsrc, vH, vW, x - 0.5, y);
    }
  }
}

/*
 * backends/numba/operators/forces.py:19-105 (compute_buoyancy_force,
 * compute_temperature_force, apply_forces). v is (H+1, W); density and
 * temperature are (H, W). The reference stores both force temporaries as
 * float32 whatever the field type (forces.py:33, :62); f32_temporaries=1 keeps
 * that rounding, 0 keeps them in float64 (used by the differentiable path).
 * Buoyancy quirk kept: rows 0 and H-1 use density[j] alone, row H gets 0.
 */
void FN(or_apply_forces)(REAL* v, long H, long W, const REAL* density, const REAL* temperature,
                         double dt, double gravity, double buoyancy_coefficient,
                         double density_coefficient, double ambient, int f32_temporaries) {
#pragma omp parallel for schedule(static)
  for (long j = 0; j < H + 1; ++j) {
    for (long i = 0; i < W; ++i) {
      double bf = 0.0, tf;
      if (j < H) {
        double d;
        if (j == 0 || j == H - 1) d = (double)density[j * W + i];
        else { REAL s = density[(j - 1) * W + i] + density[j * W + i]; d = 0.5 * (double)s; }
        bf = -density_coefficient * d * gravity;
      }
      double t;
      if (j == 0) t = (double)temperature[i];
      else if (j == H) t = (double)temperature[(H - 1) * W + i];
      else { REAL s = temperature[(j - 1) * W + i] + temperature[j * W + i]; t = 0.5 * (double)s; }
      tf = -buoyancy_coefficient * (t - ambient);
      double add;
      if (f32_temporaries) {
        float bf32 = (float)bf, tf32 = (float)tf;
        float s = bf32 + tf32;
        add = dt * (double)s;
      } else {
        add = dt * (bf + tf);
      }
      v[j * W + i] = (REAL)((double)v[j * W + i] + add);
    }
  }
}

/* forces.py:108-123 (cool_temperature) */
void FN(or_cool_temperature)(REAL* T, long H, long W, double ambient, double rate, double dt) {
  double decay = exp(-rate * dt);
#pragma omp parallel for schedule(static)
  for (long k = 0; k < H * W; ++k) T[k] = (REAL)(ambient + ((double)T[k] - ambient) * decay);
}

/* backends/numba/operators/divergence.py:4-25 (compute_divergence) */
void FN(or_divergence)(const REAL* u, const REAL* v, REAL* div, const unsigned char* fmu,
                       const unsigned char* fmv, long H, long W, double h) {
  double inv = 1.0 / h;
#pragma omp parallel for schedule(static)
  for (long j = 0; j < H; ++j) {
    for (long i = 0; i < W; ++i) {
      REAL a = u[j * (W + 1) + i + 1] * (REAL)fmu[j * (W + 1) + i + 1];
      REAL b = u[j * (W + 1) + i] * (REAL)fmu[j * (W + 1) + i];
      REAL c = v[(j + 1) * W + i] * (REAL)fmv[(j + 1) * W + i];
      REAL d = v[j * W + i] * (REAL)fmv[j * W + i];
      REAL du = a - b, dv = c - d;
      double dudx = (double)du * inv, dvdy = (double)dv * inv;
      div[j * W + i] = (REAL)(dudx + dvdy);
    }
  }
}

/* Neighbour gather shared by jacobi.py:18-21, residual.py:35-38, red_black_sor_gauss_seidel.py:19-22. */
static inline REAL FN(nbsum)(const REAL* p, const unsigned char* fmu, const unsigned char* fmv,
                             long H, long W, long j, long i) {
  REAL c = p[j * W + i];
  REAL l = fmu[j * (W + 1) + i] ? p[j * W + (i - 1 > 0 ? i - 1 : 0)] : c;
  REAL r = fmu[j * (W + 1) + i + 1] ? p[j * W + (i + 1 < W - 1 ? i + 1 : W - 1)] : c;
  REAL d = fmv[j * W + i] ? p[(j - 1 > 0 ? j - 1 : 0) * W + i] : c;
  REAL up = fmv[(j + 1) * W + i] ? p[(j + 1 < H - 1 ? j + 1 : H - 1) * W + i] : c;
  REAL s = l + r;
  s = s + d;
  s = s + up;
  return s;
}

/* backends/numba/solvers/jacobi.py:8-24 (_jacobi_kernel): one sweep src -> dst. */
void FN(or_jacobi_sweep)(const REAL* p, REAL* out, const REAL* div, const unsigned char* is_fluid,
                         const unsigned char* fmu, const unsigned char* fmv, long H, long W,
                         double alpha, double rb) {
#pragma omp parallel for schedule(static)
  for (long j = 0; j < H; ++j) {
    for (long i = 0; i < W; ++i) {
      if (!is_fluid[j * W + i]) { out[j * W + i] = p[j * W + i]; continue; }
      REAL s = FN(nbsum)(p, fmu, fmv, H, W, j, i);
      out[j * W + i] = (REAL)(((double)s + alpha * (double)div[j * W + i]) * rb);
    }
  }
}

/* red_black_sor_gauss_seidel.py:8-27 (in place; colour 0 is (i+j) even). */
void FN(or_rbsor)(REAL* p, const REAL* div, const unsigned char* is_fluid,
                  const unsigned char* fmu, const unsigned char* fmv, long H, long W,
                  double alpha, double rb, double omega, long iterations) {
  for (long it = 0; it < iterations; ++it) {
    for (int color = 0; color < 2; ++color) {
#pragma omp parallel for schedule(static)
      for (long j = 0; j < H; ++j) {
        long start = (j % 2 == 0) ? color : 1 - color;
        for (long i = start; i < W; i += 2) {
          if (!is_fluid[j * W + i]) continue;
          REAL s = FN(nbsum)(p, fmu, fmv, H, W, j, i);
          double np_ = ((double)s + alpha * (double)div[j * W + i]) * rb;
          p[j * W + i] = (REAL)((1.0 - omega) * (double)p[j * W + i] + omega * np_);
        }
      }
    }
  }
}

/* backends/numba/solvers/gauss_seidel.py:8-26 (serial lexicographic sweep). */
void FN(or_gauss_seidel)(REAL* p, const REAL* div, const unsigned char* is_fluid,
                         const unsigned char* fmu, const unsigned char* fmv, long H, long W,
                         double alpha, double rb, long iterations) {
  for (long it = 0; it < iterations; ++it)
    for (long j = 0; j < H; ++j)
      for (long i = 0; i < W; ++i) {
        if (!is_fluid[j * W + i]) continue;
        REAL s = FN(nbsum)(p, fmu, fmv, H, W, j, i);
        p[j * W + i] = (REAL)(((double)s + alpha * (double)div[j * W + i]) * rb);
      }
}

/* backends/numba/operators/residual.py:6-42 (compute_residual) */
void FN(or_residual)(const REAL* p, const REAL* div, const unsigned char* is_fluid,
                     const unsigned char* fmu, const unsigned char* fmv, long H, long W,
                     double alpha, double rb, REAL* out) {
  double beta = 1.0 / rb;
#pragma omp parallel for schedule(static)
  for (long j = 0; j < H; ++j) {
    for (long i = 0; i < W; ++i) {
      if (!is_fluid[j * W + i]) { out[j * W + i] = (REAL)0; continue; }
      REAL s = FN(nbsum)(p, fmu, fmv, H, W, j, i);
      out[j * W + i] = (REAL)(((double)s + alpha * (double)div[j * W + i]) - beta * (double)p[j * W + i]);
    }
  }
}

/*
 * backends/numba/operators/pressure_gradient.py:4-37. The outermost face
 * columns/rows are closed in every mask the reference builds
 * (common/simulation.py:103-107); an open outer face is rejected by the caller.
 */
void FN(or_pressure_gradient)(REAL* u, REAL* v, const REAL* p, const unsigned char* fmu,
                              const unsigned char* fmv, long H, long W, double rho, double h,
                              double dt) {
  double scale = dt / (rho * h);
#pragma omp parallel for schedule(static)
  for (long j = 0; j < H; ++j)
    for (long i = 0; i < W + 1; ++i) {
      long k = j * (W + 1) + i;
      if (fmu[k] && i > 0 && i < W) {
        REAL dp = p[j * W + i] - p[j * W + i - 1];
        u[k] = (REAL)((double)u[k] - scale * (double)dp);
      } else {
        u[k] = (REAL)0;
      }
    }
#pragma omp parallel for schedule(static)
  for (long j = 0; j < H + 1; ++j)
    for (long i = 0; i < W; ++i) {
      long k = j * W + i;
      if (fmv[k] && j > 0 && j < H) {
        REAL dp = p[j * W + i] - p[(j - 1) * W + i];
        v[k] = (REAL)((double)v[k] - scale * (double)dp);
      } else {
        v[k] = (REAL)0;
      }
    }
}

/* backends/numba/operators/boundaries.py:7-39 (enforce_boundary_conditions) */
void FN(or_enforce_bc)(REAL* u, REAL* v, const unsigned char* solid, long H, long W) {
#pragma omp parallel for schedule(static)
  for (long j = 0; j < H; ++j)
    for (long i = 0; i < W + 1; ++i) {
      int ls = i > 0 ? solid[j * W + i - 1] == 1 : 0;
      int rs = i < W ? solid[j * W + i] == 1 : 0;
      if (ls || rs) u[j * (W + 1) + i] = (REAL)0;
    }
#pragma omp parallel for schedule(static)
  for (long j = 0; j < H + 1; ++j)
    for (long i = 0; i < W; ++i) {
      int ts = j > 0 ? solid[(j - 1) * W + i] == 1 : 0;
      int bs = j < H ? solid[j * W + i] == 1 : 0;
      if (ts || bs) v[j * W + i] = (REAL)0;
    }
}

/* backends/numba/solvers/multigrid/transfer.py:5-36 (restrict: fluid-children mean) */
void FN(or_restrict_avg)(const REAL* fine, const unsigned char* fluid, long H, long W,
                         REAL* coarse, long Hc, long Wc) {
#pragma omp parallel for schedule(static)
  for (long J = 0; J < Hc; ++J)
    for (long I = 0; I < Wc; ++I) {
      double total = 0.0;
      long count = 0;
      for (int dj = 0; dj < 2; ++dj)
        for (int di = 0; di < 2; ++di) {
          long jj = 2 * J + dj, ii = 2 * I + di;
          if (fluid[jj * W + ii]) { total += (double)fine[jj * W + ii]; ++count; }
        }
      coarse[J * Wc + I] = count > 0 ? (REAL)(total / (double)count) : (REAL)0;
    }
}

/* transfer.py:38-72 (prolong: clamped bilinear sample of the coarse field) */
void FN(or_prolong)(const REAL* coarse, long Hc, long Wc, const unsigned char* fluid, long H,
                    long W, REAL* fine) {
#pragma omp parallel for schedule(static)
  for (long j = 0; j < H; ++j)
    for (long i = 0; i < W; ++i) {
      if (!fluid[j * W + i]) { fine[j * W + i] = (REAL)0; continue; }
      double xc = ((double)i + 0.5) * 0.5, yc = ((double)j + 0.5) * 0.5;
      fine[j * W + i] = (REAL)FN(sample)(coarse, Hc, Wc, xc - 0.5, yc - 0.5);
    }
}

/* common/emitters.py:6-35, :37-66 (Numba emitter path; approach 0 hard, 1 linear, 2 quadratic, 3 gaussian) */
void FN(or_emit_scalar)(REAL* field, long H, long W, double value, double dt, double px,
                        double py, double radius, int approach) {
  long x_min = (long)(px - radius - 1.0); if (x_min < 0) x_min = 0;
  long x_max = (long)(px + radius + 2.0); if (x_max > W) x_max = W;
  long y_min = (long)(py - radius - 1.0); if (y_min < 0) y_min = 0;
  long y_max = (long)(py + radius + 2.0); if (y_max > H) y_max = H;
  for (long y = y_min; y < y_max; ++y)
    for (long x = x_min; x < x_max; ++x) {
      double dx = (double)x - px, dy = (double)y - py;
      double dist = sqrt(dx * dx + dy * dy);
      if (dist < radius) {
        double f;
        if (approach == 0) f = 1.0;
        else if (approach == 1) f = 1.0 - dist / radius;
        else if (approach == 2) f = 1.0 - (dist / radius) * (dist / radius);
        else { double s = radius / 3.0; f = exp(-0.5 * (dist / s) * (dist / s)); }
        field[y * W + x] = (REAL)((double)field[y * W + x] + value * f * dt);
      }
    }
}

/*
 * Plume source (no reference counterpart; the benchmark scenes' source):
 * cells whose centre ((i+.5), (j+.5)) lies strictly inside the disc get
 * density = dens_value; v faces at ((i+.5), j) inside get v_value + noise;
 * u faces at (i, (j+.5)) inside get noise. Coordinates are in cells.
 */
void FN(or_plume_source)(REAL* density, REAL* u, REAL* v, long H, long W, double cx, double cy,
                         double radius, double dens_value, double v_value, double noise_amp,
                         unsigned long long seed, long step) {
  double r2 = radius * radius;
  for (long j = 0; j < H; ++j)
    for (long i = 0; i < W; ++i) {
      double dx = (double)i + 0.5 - cx, dy = (double)j + 0.5 - cy;
      if (dx * dx + dy * dy < r2) density[j * W + i] = (REAL)dens_value;
    }
  for (long j = 0; j < H + 1; ++j)
    for (long i = 0; i < W; ++i) {
      double dx = (double)i + 0.5 - cx, dy = (double)j - cy;
      if (dx * dx + dy * dy < r2)
        v[j * W + i] = (REAL)(v_value + sg_noise(seed, step, 1, j, i, noise_amp));
    }
  for (long j = 0; j < H; ++j)
    for (long i = 0; i < W + 1; ++i) {
      double dx = (double)i - cx, dy = (double)j + 0.5 - cy;
      if (dx * dx + dy * dy < r2)
        u[j * (W + 1) + i] = (REAL)sg_noise(seed, step, 0, j, i, noise_amp);
    }
}

/* ------------------------------------------------------------------------ */
/* Convergent geometric multigrid pieces (no reference counterpart).         */
/* Operator A p = sum_open (p - p_nb) on fluid cells; residual r = b - A p,  */
/* which equals residual.py:39-40 with b = alpha*div.                        */
/* ------------------------------------------------------------------------ */

/* r = b - A p on fluid cells, 0 elsewhere. */
void FN(or_gmg_residual)(const REAL* p, const REAL* b, const unsigned char* fluid,
                         const unsigned char* fmu, const unsigned char* fmv, long H, long W,
                         REAL* r) {
#pragma omp parallel for schedule(static)
  for (long j = 0; j < H; ++j)
    for (long i = 0; i < W; ++i) {
      long k = j * W + i;
      if (!fluid[k]) { r[k] = (REAL)0; continue; }
      REAL c = p[k];
      REAL acc = b[k];
      if (fmu[j * (W + 1) + i]) acc += p[k - 1] - c;
      if (fmu[j * (W + 1) + i + 1]) acc += p[k + 1] - c;
      if (fmv[j * W + i]) acc += p[k - W] - c;
      if (fmv[(j + 1) * W + i]) acc += p[k + W] - c;
      r[k] = acc;
    }
}

/* Red-black Gauss-Seidel with over-relaxation omega and the exact diagonal. */
void FN(or_gmg_rbgs)(REAL* p, const REAL* b, const unsigned char* fluid,
                     const unsigned char* fmu, const unsigned char* fmv, long H, long W,
                     double omega, long sweeps) {
  for (long s = 0; s < sweeps; ++s)
    for (int color = 0; color < 2; ++color) {
#pragma omp parallel for schedule(static)
      for (long j = 0; j < H; ++j)
        for (long i = (j + color) & 1; i < W; i += 2) {
          long k = j * W + i;
          if (!fluid[k]) continue;
          REAL acc = b[k];
          int n = 0;
          if (fmu[j * (W + 1) + i]) { acc += p[k - 1]; ++n; }
          if (fmu[j * (W + 1) + i + 1]) { acc += p[k + 1]; ++n; }
          if (fmv[j * W + i]) { acc += p[k - W]; ++n; }
          if (fmv[(j + 1) * W + i]) { acc += p[k + W]; ++n; }
          if (n == 0) continue;
          REAL gs = acc / (REAL)n;
          p[k] = p[k] + (REAL)omega * (gs - p[k]);
        }
    }
}

/*
 * Bilinear cell-centred prolongation weights of fine cell (j,i) onto the
 * coarse grid: the home cell (j>>1, i>>1) takes 9/16, the x and y neighbours
 * towards the fine cell 3/16 each, the diagonal 1/16. Indices are clamped to
 * the coarse grid; a candidate that is not fluid is replaced by the home cell.
 */
static inline void FN(gmg_pweights)(long j, long i, long Hc, long Wc, const unsigned char* cfluid,
                                    long cj[4], long ci[4]) {
  long J = j >> 1, I = i >> 1;
  long X = I + ((i & 1) ? 1 : -1), Y = J + ((j & 1) ? 1 : -1);
  if (X < 0) X = 0; if (X > Wc - 1) X = Wc - 1;
  if (Y < 0) Y = 0; if (Y > Hc - 1) Y = Hc - 1;
  cj[0] = J; ci[0] = I;
  cj[1] = J; ci[1] = X;
  cj[2] = Y; ci[2] = I;
  cj[3] = Y; ci[3] = X;
  for (int q = 1; q < 4; ++q)
    if (!cfluid[cj[q] * Wc + ci[q]]) { cj[q] = J; ci[q] = I; }
}

/* e_fine += P e_coarse on fluid fine cells. */
void FN(or_gmg_prolong_add)(const REAL* ec, const unsigned char* cfluid, long Hc, long Wc,
                            REAL* e, const unsigned char* fluid, long H, long W) {
  static const double w[4] = {9.0 / 16.0, 3.0 / 16.0, 3.0 / 16.0, 1.0 / 16.0};
#pragma omp parallel for schedule(static)
  for (long j = 0; j < H; ++j)
    for (long i = 0; i < W; ++i) {
      if (!fluid[j * W + i]) continue;
      long cj[4], ci[4];
      FN(gmg_pweights)(j, i, Hc, Wc, cfluid, cj, ci);
      REAL acc = (REAL)0;
      for (int q = 0; q < 4; ++q) acc += (REAL)w[q] * ec[cj[q] * Wc + ci[q]];
      e[j * W + i] += acc;
    }
}

/* b_coarse = P^T r (full weighting: the transpose of the prolongation). */
void FN(or_gmg_restrict_fw)(const REAL* r, const unsigned char* fluid, long H, long W,
                            REAL* bc, const unsigned char* cfluid, long Hc, long Wc) {
  static const double w[4] = {9.0 / 16.0, 3.0 / 16.0, 3.0 / 16.0, 1.0 / 16.0};
#pragma omp parallel for schedule(static)
  for (long J = 0; J < Hc; ++J)
    for (long I = 0; I < Wc; ++I) {
      REAL acc = (REAL)0;
      if (cfluid[J * Wc + I]) {
        for (long j = 2 * J - 2; j <= 2 * J + 3; ++j) {
          if (j < 0 || j >= H) continue;
          for (long i = 2 * I - 2; i <= 2 * I + 3; ++i) {
            if (i < 0 || i >= W || !fluid[j * W + i]) continue;
            long cj[4], ci[4];
            FN(gmg_pweights)(j, i, Hc, Wc, cfluid, cj, ci);
            for (int q = 0; q < 4; ++q)
              if (cj[q] == J && ci[q] == I) acc += (REAL)w[q] * r[j * W + i];
          }
        }
      }
      bc[J * Wc + I] = acc;
    }
}
