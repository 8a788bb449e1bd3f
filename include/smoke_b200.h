/*
 * smoke_b200 -- C ABI of the B200 (sm_100a) smoke-simulation step.
 *
 * Every entry point takes plain device pointers, sizes and row strides (in
 * elements), a dtype code, and a CUDA stream (cudaStream_t passed as void*).
 * Calls are stream-ordered and asynchronous unless stated otherwise; none
 * allocates device memory except where "allocates" is written below. Return
 * value: SG_OK (0) or an SG_ERR_* code; sg_last_error() gives the message of the
 * calling thread's last failure. No C++ exception crosses this boundary.
 *
 * Arrays are row-major [row j = y][column i = x]. For a grid of H rows and W
 * columns: cell fields are H x W, u faces H x (W+1), v faces (H+1) x W
 * (reference: src/cfd/common/simulation.py:76-84).
 *
 * Masks (uint8, 0/1) are selected by a mask mode:
 *   SG_MASK_PLANES  explicit planes, as the reference passes them;
 *   SG_MASK_OPEN    all interior faces open, outer faces closed (what
 *                   SmokeSimulation2D builds at construction,
 *                   common/simulation.py:102-113); planes may be NULL;
 *   SG_MASK_RING    faces of a box whose outermost cells are solid
 *                   (the solid ring of simulation.py:126-131); planes may be NULL.
 * The outermost face columns/rows must be closed in SG_MASK_PLANES mode, as every
 * mask the reference builds is (simulation.py:103-107).
 *
 * Reference citations name files of LCEBurton/python-game-engine under src/cfd/.
 */
#ifndef SMOKE_B200_H
#define SMOKE_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SG_F32 0
#define SG_F64 1

#define SG_MASK_PLANES 0
#define SG_MASK_OPEN 1
#define SG_MASK_RING 2
#define SG_MASK_NONE 3 /* enforce_boundary_conditions only: no solid cells */

#define SG_OK 0
#define SG_ERR_ARG 1          /* null pointer, bad size, stride, mode or parameter */
#define SG_ERR_DTYPE 2        /* unsupported dtype code */
#define SG_ERR_CUDA 3         /* a CUDA runtime call failed */
#define SG_ERR_NOT_CONVERGED 4 /* tolerance not reached within the cycle/iteration cap */
#define SG_ERR_NONFINITE 5    /* a NaN or Inf was detected in a residual norm */
#define SG_ERR_WORKSPACE 6    /* workspace missing or too small */
#define SG_ERR_CAPACITY 7     /* size above a fixed capacity */

const char* sg_version(void);
/* Message of the calling thread's last failing call ("" if none). */
const char* sg_last_error(void);
/* Number of kernel launches this library has issued since it was loaded (all threads). */
uint64_t sg_launch_count(void);

/* ---------------------------------------------------------------- operators */

/* backends/numba/operators/advection.py:112-128 (advect_scalar_field) and the
 * dissipation of common/simulation.py:232 fused in: dst = round(sample) * dissipation
 * in the field's dtype (pass 1.0 for none). u is u_rows x u_cols, v is v_rows x v_cols
 * (the reference samples them with clamping to their own shapes). is_fluid: H x W. */
int sg_advect_scalar(int dtype, int64_t H, int64_t W, const void* src, int64_t ld_src, void* dst,
                     int64_t ld_dst, const void* u, int64_t u_rows, int64_t u_cols, int64_t ld_u,
                     const void* v, int64_t v_rows, int64_t v_cols, int64_t ld_v, int mask_mode,
                     const uint8_t* is_fluid, int64_t ld_fluid, double dt, double cell_size,
                     double dissipation, void* stream);

/* advection.py:130-154 (advect_velocity_u). u is u_rows x u_cols, v is v_rows x v_cols. */
int sg_advect_velocity_u(int dtype, int64_t u_rows, int64_t u_cols, const void* u_src, int64_t ld_us,
                         void* u_dst, int64_t ld_ud, const void* v, int64_t v_rows, int64_t v_cols,
                         int64_t ld_v, int mask_mode, const uint8_t* fmu, int64_t ld_fmu, double dt,
                         double cell_size, void* stream);

/* advection.py:156-180 (advect_velocity_v). */
int sg_advect_velocity_v(int dtype, int64_t v_rows, int64_t v_cols, const void* v_src, int64_t ld_vs,
                         void* v_dst, int64_t ld_vd, const void* u, int64_t u_rows, int64_t u_cols,
                         int64_t ld_u, int mask_mode, const uint8_t* fmv, int64_t ld_fmv, double dt,
                         double cell_size, void* stream);

/* Both of the above in one launch on MAC-shaped fields (common/simulation.py:280-286:
 * both read the old u and v). */
int sg_advect_velocity(int dtype, int64_t H, int64_t W, const void* u_src, int64_t ld_us, void* u_dst,
                       int64_t ld_ud, const void* v_src, int64_t ld_vs, void* v_dst, int64_t ld_vd,
                       int mask_mode, const uint8_t* fmu, int64_t ld_fmu, const uint8_t* fmv,
                       int64_t ld_fmv, double dt, double cell_size, void* stream);

/* float32 fields advected in float32 arithmetic (advection.py:112-180: same backtrace,
 * clamped bilinear sampling, masks and dissipation). The reference evaluates positions and
 * weights in float64; here the backtrace offset -vel * dt / h is taken relative to the
 * sampling point's cell, so the weights keep float32's relative precision, and the result
 * equals the reference's up to rounding (not bit for bit). Velocity fields in MAC shapes
 * (H x (W+1), (H+1) x W); masks as for sg_advect_velocity / sg_advect_scalar. */
int sg_advect_velocity_f32(int64_t H, int64_t W, const void* u_src, int64_t ld_us, void* u_dst, int64_t ld_ud,
                           const void* v_src, int64_t ld_vs, void* v_dst, int64_t ld_vd, int mask_mode,
                           const uint8_t* fmu, int64_t ld_fmu, const uint8_t* fmv, int64_t ld_fmv, double dt,
                           double cell_size, void* stream);
int sg_advect_scalar_f32(int64_t H, int64_t W, const void* src, int64_t ld_src, void* dst, int64_t ld_dst,
                         const void* u, int64_t ld_u, const void* v, int64_t ld_v, int mask_mode,
                         const uint8_t* is_fluid, int64_t ld_fluid, double dt, double cell_size, double dissipation,
                         void* stream);

/* backends/numba/operators/forces.py:78-105 (apply_forces). v is (H+1) x W; density and
 * temperature are H x W. temperature may be NULL (treated as ambient everywhere).
 * f32_temporaries=1 rounds both force terms to float32 as the reference does
 * (forces.py:33, :62); 0 keeps them in the field's dtype. */
int sg_apply_forces(int dtype, int64_t H, int64_t W, void* v, int64_t ld_v, const void* density,
                    int64_t ld_d, const void* temperature, int64_t ld_t, double dt, double gravity,
                    double buoyancy_coefficient, double density_coefficient, double ambient_temperature,
                    int f32_temporaries, void* stream);

/* forces.py:108-123 (cool_temperature). */
int sg_cool_temperature(int dtype, int64_t H, int64_t W, void* temperature, int64_t ld_t, double ambient,
                        double cooling_rate, double dt, void* stream);

/* backends/numba/operators/divergence.py:4-25 (compute_divergence). */
int sg_compute_divergence(int dtype, int64_t H, int64_t W, const void* u, int64_t ld_u, const void* v,
                          int64_t ld_v, void* div, int64_t ld_div, int mask_mode, const uint8_t* fmu,
                          int64_t ld_fmu, const uint8_t* fmv, int64_t ld_fmv, double cell_size,
                          void* stream);

/* backends/numba/operators/residual.py:6-42 (compute_residual). If sumsq (device, one
 * double) is non-NULL, the sum over fluid cells of residual^2 (evaluated in double) is
 * ADDED to it. */
int sg_compute_residual(int dtype, int64_t H, int64_t W, const void* p, int64_t ld_p, const void* div,
                        int64_t ld_div, int mask_mode, const uint8_t* is_fluid, int64_t ld_fluid,
                        const uint8_t* fmu, int64_t ld_fmu, const uint8_t* fmv, int64_t ld_fmv,
                        double alpha, double reciprocal_beta, void* out, int64_t ld_out, double* sumsq,
                        void* stream);

/* backends/numba/operators/pressure_gradient.py:4-37 (apply_pressure_gradient). */
int sg_apply_pressure_gradient(int dtype, int64_t H, int64_t W, void* u, int64_t ld_u, void* v,
                               int64_t ld_v, const void* p, int64_t ld_p, int mask_mode, const uint8_t* fmu,
                               int64_t ld_fmu, const uint8_t* fmv, int64_t ld_fmv, double fluid_density,
                               double cell_size, double dt, void* stream);

/* backends/numba/operators/boundaries.py:7-39 (enforce_boundary_conditions).
 * solid_mode: SG_MASK_PLANES (solid plane H x W), SG_MASK_RING, or SG_MASK_NONE. */
int sg_enforce_boundary_conditions(int dtype, int64_t H, int64_t W, void* u, int64_t ld_u, void* v,
                                   int64_t ld_v, int solid_mode, const uint8_t* solid, int64_t ld_s,
                                   void* stream);

/* apply_pressure_gradient followed by enforce_boundary_conditions in one pass over the
 * faces (common/simulation.py:244-249). */
int sg_project(int dtype, int64_t H, int64_t W, void* u, int64_t ld_u, void* v, int64_t ld_v,
               const void* p, int64_t ld_p, int mask_mode, const uint8_t* fmu, int64_t ld_fmu,
               const uint8_t* fmv, int64_t ld_fmv, int solid_mode, const uint8_t* solid, int64_t ld_s,
               double fluid_density, double cell_size, double dt, void* stream);

/* The substep's tail in one pass (simulation.py:244-265): sg_project of (u_in, v_in) into
 * (u_out, v_out) (out of place; the inputs are not changed), then sg_compute_divergence of
 * the projected field into div and sg_compute_residual of p with that divergence into res.
 * Every value equals the three separate passes'. No single reference function: it fuses
 * apply_pressure_gradient + enforce_boundary_conditions + compute_divergence +
 * compute_residual. */
int sg_project_metrics(int dtype, int64_t H, int64_t W, const void* u_in, int64_t ld_ui, const void* v_in,
                       int64_t ld_vi, void* u_out, int64_t ld_uo, void* v_out, int64_t ld_vo, const void* p,
                       int64_t ld_p, int mask_mode, const uint8_t* fmu, int64_t ld_fmu, const uint8_t* fmv,
                       int64_t ld_fmv, const uint8_t* is_fluid, int64_t ld_fluid, int solid_mode, const uint8_t* solid,
                       int64_t ld_s, double fluid_density, double cell_size, double dt, double alpha,
                       double reciprocal_beta, void* div, int64_t ld_div, void* res, int64_t ld_res, void* stream);

/* Float32 fields in float32 arithmetic (no counterpart in the reference, whose kernels form
 * these terms in float64; results equal the reference's up to rounding, 1e-5 of the fields'
 * magnitude in the tests): the buoyancy force of sg_apply_forces (forces.py:19-105, the
 * reference's face averaging) and the projection tail of sg_project_metrics
 * (pressure_gradient.py:4-37, boundaries.py:7-39, divergence.py:4-25, residual.py:6-42).
 * Same arguments as those entries without the dtype (and without f32_temporaries). Fields
 * below 2^31 elements. */
int sg_apply_forces_f32(int64_t H, int64_t W, void* v, int64_t ld_v, const void* density, int64_t ld_d,
                        const void* temperature, int64_t ld_t, double dt, double gravity, double buoyancy_coefficient,
                        double density_coefficient, double ambient_temperature, void* stream);
int sg_project_metrics_f32(int64_t H, int64_t W, const void* u_in, int64_t ld_ui, const void* v_in, int64_t ld_vi,
                           void* u_out, int64_t ld_uo, void* v_out, int64_t ld_vo, const void* p, int64_t ld_p,
                           int mask_mode, const uint8_t* fmu, int64_t ld_fmu, const uint8_t* fmv, int64_t ld_fmv,
                           const uint8_t* is_fluid, int64_t ld_fluid, int solid_mode, const uint8_t* solid,
                           int64_t ld_s, double fluid_density, double cell_size, double dt, double alpha,
                           double reciprocal_beta, void* div, int64_t ld_div, void* res, int64_t ld_res,
                           void* stream);

/* common/emitters.py:37-66 (_apply_scalar_field_numba); approach 0 hard_cutoff,
 * 1 linear, 2 quadratic, 3 gaussian (emitters.py:6-35). */
int sg_emit_scalar(int dtype, int64_t H, int64_t W, void* field, int64_t ld, double value, double dt,
                   double pos_x, double pos_y, double radius, int approach, void* stream);

/* Plume sources of the benchmark scenes (no reference counterpart; the reference's
 * emitters add, these overwrite). sources: HOST array of n_sources (<= 32) x 6 doubles
 * (cx, cy, radius, density_value, v_value, noise_amp) in cell units, copied into the
 * launch parameters (the array may be reused when the call returns); the launch covers
 * the union of the sources' bounding boxes only. Cells whose
 * centre (i+.5, j+.5) is strictly inside get density; v faces at (i+.5, j) get
 * v_value + noise, u faces at (i, j+.5) get noise; noise is uniform in
 * [-amp, amp), keyed by (seed, step, component, row, column). */
int sg_plume_sources(int dtype, int64_t H, int64_t W, void* density, int64_t ld_d, void* u, int64_t ld_u,
                     void* v, int64_t ld_v, int n_sources, const double* sources, uint64_t seed,
                     int64_t step, void* stream);

/* common/simulation.py:103-108 / multigrid/masks.py:30-74: face masks and is_fluid
 * from a solid plane (any output may be NULL). */
int sg_build_masks(int64_t H, int64_t W, const uint8_t* solid, int64_t ld_s, uint8_t* fmu, int64_t ld_fmu,
                   uint8_t* fmv, int64_t ld_fmv, uint8_t* is_fluid, int64_t ld_fluid, void* stream);

/* Bounds-check build (lib/libsmoke_b200_bc.so, compiled with -DSG_BOUNDS_CHECK=1): the
 * tiled kernels check their index arithmetic before each access, skip an access that fails
 * and record the source line of the first failure per compilation unit; nothing traps.
 * sg_bounds_check reports the first recorded line (0: none) and its unit (0 operators,
 * 1 gmg, 2 batch, 3 rbsor_split, 4 advect_fast, 5 adjoint, 6 metrics; -1: none) and, with
 * clear != 0, resets the records. sg_bounds_check_enabled: 1 in that build, 0 otherwise (where
 * sg_bounds_check always reports none). No counterpart in the reference. */
int sg_bounds_check_enabled(void);
int sg_bounds_check(unsigned int* first_line, int* unit, int clear);

/* ---------------------------------------------------------------- reference solvers */

/* backends/numba/solvers/jacobi.py:8-52: `iterations` ping-pong sweeps. scratch: device
 * buffer of H*W elements of dtype (row stride W); the result always ends in p. */
int sg_jacobi_solve(int dtype, int64_t H, int64_t W, void* p, int64_t ld_p, const void* div,
                    int64_t ld_div, int mask_mode, const uint8_t* fmu, int64_t ld_fmu, const uint8_t* fmv,
                    int64_t ld_fmv, double alpha, double reciprocal_beta, int iterations, void* scratch,
                    void* stream);

/* Same solve as sg_jacobi_solve for callers that cannot allocate device memory: a game
 * loop or real-time host that must not call cudaMalloc during a frame (an allocation can
 * synchronise the device and stall the frame), or a host that runs under a fixed device
 * memory budget set at start-up. No counterpart in the reference (its Jacobi allocates a
 * temporary per call, jacobi.py:45).
 * The ping-pong buffer is a file-scope __device__ array of SG_JACOBI_NOALLOC_MAX_BYTES
 * bytes that every GPU loading this library holds until exit, so H * W * sizeof(dtype)
 * must not exceed it (1024 x 1024 float32, 724 x 724 float64); larger grids return
 * SG_ERR_CAPACITY. The first call on each device looks the array's address up
 * (cudaGetSymbolAddress) with that device current; make that first call before any
 * stream capture. The address is kept for the life of the process: after a
 * cudaDeviceReset on a device, do not call this entry point on that device again until
 * the library has been unloaded and loaded again. All calls share the one array: calls that overlap on the GPU (other
 * streams, other host threads) race and must be serialised by the caller. Nothing in
 * the array needs clearing: the first sweep writes every cell before it is read.
 * Allocates nothing and calls no allocating routine. */
#define SG_JACOBI_NOALLOC_MAX_BYTES (4u << 20)
int sg_jacobi_solve_noalloc(int dtype, int64_t H, int64_t W, void* p, int64_t ld_p, const void* div,
                            int64_t ld_div, int mask_mode, const uint8_t* fmu, int64_t ld_fmu,
                            const uint8_t* fmv, int64_t ld_fmv, double alpha, double reciprocal_beta,
                            int iterations, void* stream);

/* backends/numba/solvers/red_black_sor_gauss_seidel.py:8-42: in place, colour 0 = (i+j) even.
 * omega as given (the caller resolves the reference's auto-omega rule). */
int sg_rbsor_solve(int dtype, int64_t H, int64_t W, void* p, int64_t ld_p, const void* div, int64_t ld_div,
                   int mask_mode, const uint8_t* fmu, int64_t ld_fmu, const uint8_t* fmv, int64_t ld_fmv,
                   double alpha, double reciprocal_beta, double omega, int iterations, void* stream);

/* Red-black SOR on a checkerboard-split layout (red_black_sor_gauss_seidel.py:8-42; the
 * tolerance loop has no reference counterpart: the reference runs a fixed sweep count).
 * Cell (j, i) of colour c = (i + j) & 1 lives in plane c at row j, column i >> 1, so each
 * colour streams contiguously. The iterates equal sg_rbsor_solve's bit for bit.
 * Workspace (256-byte aligned, sg_rbsor_split_workspace_bytes): two state buffers of two
 * planes each, the two divergence planes and the residual partial sums.
 *   pack:   which = 0 copies the pressure into the state, 1 the divergence
 *   sweeps: `iterations` sweeps (colour 0 then 1) on the state; variant 0 launches one
 *           streaming kernel per half sweep, variant 1 sweeps 32 x 64 tiles staged in shared
 *           memory up to 4 sweeps per launch (same iterates), -1 picks the tiles while
 *           2 * H * W * sizeof(dtype) <= 8 MiB (L2-resident, launch-bound) and the
 *           streaming launches above (bandwidth-bound)
 *   sumsq:  *out (device) = sum over fluid cells of the squared reference residual
 *           (residual.py:39-40) of the state, or of p = 0 when zero_p is set
 *   unpack: the state back to a natural-layout field
 *   tol_solve: pack, then sweeps in chunks of check_every until ||r(p)|| <= tol ||r(0)||
 *           (fluid cells) or max_iterations, then unpack into p; synchronises the stream
 *           after every chunk to read the residual. Returns SG_ERR_NOT_CONVERGED (p still
 *           written, *out_iterations / *out_relres set) when the tolerance is not reached. */
int64_t sg_rbsor_split_workspace_bytes(int dtype, int64_t H, int64_t W);
int sg_rbsor_split_pack(int dtype, int64_t H, int64_t W, const void* src, int64_t ld_src, int which,
                        void* workspace, int64_t workspace_bytes, void* stream);
int sg_rbsor_split_unpack(int dtype, int64_t H, int64_t W, const void* workspace, int64_t workspace_bytes,
                          void* dst, int64_t ld_dst, void* stream);
int sg_rbsor_split_sweeps(int dtype, int64_t H, int64_t W, void* workspace, int64_t workspace_bytes,
                          int mask_mode, const uint8_t* fmu, int64_t ld_fmu, const uint8_t* fmv,
                          int64_t ld_fmv, double alpha, double reciprocal_beta, double omega,
                          int64_t iterations, int variant, void* stream);
int sg_rbsor_split_sumsq(int dtype, int64_t H, int64_t W, void* workspace, int64_t workspace_bytes,
                         int mask_mode, const uint8_t* fmu, int64_t ld_fmu, const uint8_t* fmv,
                         int64_t ld_fmv, double alpha, double reciprocal_beta, int zero_p, double* out,
                         void* stream);
int sg_rbsor_tol_solve(int dtype, int64_t H, int64_t W, void* p, int64_t ld_p, const void* div,
                       int64_t ld_div, int mask_mode, const uint8_t* fmu, int64_t ld_fmu,
                       const uint8_t* fmv, int64_t ld_fmv, double alpha, double reciprocal_beta,
                       double omega, double tol, int64_t max_iterations, int64_t check_every,
                       int variant, void* workspace, int64_t workspace_bytes, int64_t* out_iterations,
                       double* out_relres, void* stream);

/* Mixed-precision red-black SOR (no reference counterpart): float64 iterative refinement
 * around the split-layout float32 sweeps, for a float32 pressure and divergence that must
 * reach a residual below float32's floor (~1e-4 relative on a 512^2 plume). The pressure is
 * accumulated in float64; each refinement forms the float64 reference residual
 * (residual.py:39-40) and solves A e = float32(r) from e = 0 with float32 sweeps
 * (red_black_sor_gauss_seidel.py:8-27 with alpha = 1) in chunks of check_every, to
 * max(1e-3, tol / (2 relres)) (at most 0.5) or until three chunks in a row gain < 1 %;
 * then p += e. Stops at ||r(p)|| <= tol ||r(0)|| (fluid cells) or max_iterations sweeps.
 * variant as for sg_rbsor_split_sweeps. Workspace: sg_rbsor_mixed_workspace_bytes
 * (256-byte aligned). Synchronises the stream after every chunk. SG_ERR_NOT_CONVERGED when
 * the tolerance is not reached (p written). */
int64_t sg_rbsor_mixed_workspace_bytes(int64_t H, int64_t W);
int sg_rbsor_mixed_solve(int64_t H, int64_t W, void* p, int64_t ld_p, const void* div, int64_t ld_div,
                         int mask_mode, const uint8_t* fmu, int64_t ld_fmu, const uint8_t* fmv,
                         int64_t ld_fmv, double alpha, double reciprocal_beta, double omega, double tol,
                         int64_t max_iterations, int64_t check_every, int variant, void* workspace,
                         int64_t workspace_bytes, int64_t* out_iterations, double* out_relres,
                         int64_t* out_refinements, void* stream);

/* backends/numba/solvers/gauss_seidel.py:8-48 (lexicographic order), run as an
 * anti-diagonal wavefront in one thread block; intended for small grids. */
int sg_gauss_seidel_solve(int dtype, int64_t H, int64_t W, void* p, int64_t ld_p, const void* div,
                          int64_t ld_div, int mask_mode, const uint8_t* fmu, int64_t ld_fmu,
                          const uint8_t* fmv, int64_t ld_fmv, double alpha, double reciprocal_beta,
                          int iterations, void* stream);

/* multigrid/transfer.py:5-36 (restrict: mean of the fluid children) with the coarse
 * rhs division of multigrid/solver.py:124-125 fused (coarse = round(mean) / round(divisor)
 * in dtype; pass 1.0 for none). */
int sg_mg_restrict_average(int dtype, int64_t H, int64_t W, const void* fine, int64_t ld_f, int mask_mode,
                           const uint8_t* is_fluid, int64_t ld_fluid, void* coarse, int64_t ld_c,
                           int64_t Hc, int64_t Wc, double divisor, void* stream);

/* multigrid/transfer.py:38-72 (prolong). accumulate=0 writes fine = P coarse;
 * accumulate=1 performs the `pressure += correction` of multigrid/solver.py:133-134
 * (fine = fine + round(P coarse)). */
int sg_mg_prolong(int dtype, int64_t Hc, int64_t Wc, const void* coarse, int64_t ld_c, int64_t H, int64_t W,
                  int mask_mode, const uint8_t* is_fluid, int64_t ld_fluid, void* fine, int64_t ld_f,
                  int accumulate, void* stream);

/* multigrid/masks.py:3-27 (any solid child makes the coarse cell solid). */
int sg_mg_coarsen_solid(int64_t H, int64_t W, const uint8_t* solid, int64_t ld_s, uint8_t* coarse,
                        int64_t ld_c, void* stream);

/* ---------------------------------------------------------------- convergent multigrid */
/*
 * Geometric multigrid for A p = b with A p = sum over open faces (p - p_nb) on fluid
 * cells and b = alpha * div (so r = b - A p equals residual.py:39-40). No reference
 * counterpart: the reference V-cycle (multigrid/solver.py) does not converge to
 * tight tolerances. Any-fluid 2x2 coarsening, red-black Gauss-Seidel smoother with
 * over-relaxation, full-weighting restriction (transpose of bilinear prolongation),
 * exact coarsest solve (pseudo-inverse). precision: SG_GMG_FP32, SG_GMG_FP64, or
 * SG_GMG_MIXED (FP64 fine residual and pressure accumulation, FP32 cycles, FP64
 * coarsest solve).
 */
#define SG_GMG_FP32 0
#define SG_GMG_FP64 1
#define SG_GMG_MIXED 2

typedef struct sg_gmg_plan sg_gmg_plan;

/* Copy the last solve's relative residual (a double) to `dst` (host-pinned or device
 * memory) on `stream`, without synchronising. */
int sg_gmg_relres_async(sg_gmg_plan* plan, double* dst, void* stream);

/* Host-side planning (allocates host memory only). The masks are HOST arrays
 * (NULL in SG_MASK_OPEN / SG_MASK_RING modes). cycle: 0 = V, 1 = W. */
int sg_gmg_plan_create(sg_gmg_plan** plan, int64_t H, int64_t W, int mask_mode, const uint8_t* is_fluid,
                       const uint8_t* fmu, const uint8_t* fmv, int coarsest, double omega, int pre_sweeps,
                       int post_sweeps, int cycle, int precision);
void sg_gmg_plan_destroy(sg_gmg_plan* plan);
int64_t sg_gmg_workspace_bytes(const sg_gmg_plan* plan);
int sg_gmg_num_levels(const sg_gmg_plan* plan);
/* Copy the plan's level masks and coarsest operator into a caller-provided device
 * workspace of sg_gmg_workspace_bytes() bytes (256-byte aligned) and reset the solve
 * statistics. Synchronises stream. */
int sg_gmg_bind(sg_gmg_plan* plan, void* workspace, void* stream);
/* Solve in place from the current p (p is float32 for SG_GMG_FP32, float64 otherwise;
 * div is float32 or float64 as div_dtype says) until ||b - A p|| / ||b|| <= tol or
 * max_cycles (< 128) cycles, without host synchronisation: the first call for a given
 * (p, div) pair captures the solve into a CUDA graph (instantiated once, kept by the
 * plan) whose cycles run inside a conditional WHILE node; the convergence test runs on
 * the device after every cycle. Read the outcome with sg_gmg_stats. */
int sg_gmg_solve_async(sg_gmg_plan* plan, void* p, int64_t ld_p, const void* div, int64_t ld_div, int div_dtype,
                       double alpha, double tol, int max_cycles, void* stream);
/* As sg_gmg_solve_async from the initial guess p = 0: p is written, never read (the
 * reference zeroes the pressure before every solve, simulation.py:310; this saves the
 * first residual pass). */
int sg_gmg_solve_from_zero_async(sg_gmg_plan* plan, void* p, int64_t ld_p, const void* div, int64_t ld_div,
                                 int div_dtype, double alpha, double tol, int max_cycles, void* stream);
/* Remove the mean of alpha * div over the fluid cells from the rhs before solving (on = 1)
 * or not (0, the default). The pressure equation with closed walls is a Neumann problem:
 * its rhs must sum to zero, which a divergence does exactly only in exact arithmetic; the
 * float rounding of that sum leaves a constant component that no pressure removes, and it
 * sets a floor under the relative residual (near 1e-10 for a float32 state at 2048^2).
 * No counterpart in the reference. */
int sg_gmg_set_remove_mean(sg_gmg_plan* plan, int on);
/* Cycles per refinement step, 1..8 (default 1). With 1, a plan whose fine level runs the
 * fused kernels corrects p and updates the fine-precision residual inside every cycle's
 * post-smoothing kernel. With k >= 2 (classical iterative refinement) each step of the
 * tolerance loop runs k cycles on the cycle-precision correction from zero, then p += e and
 * one fine-precision residual pass; the cycle count grows by k per step. No counterpart in
 * the reference. */
int sg_gmg_set_inner_cycles(sg_gmg_plan* plan, int inner);
/* Outcome of the last solve (synchronises stream): cycles run, last relative residual,
 * status (1 converged, 2 cycle cap reached, 3 non-finite residual) and the number of
 * cycles run by all solves since sg_gmg_bind. Any output may be NULL. */
int sg_gmg_stats(sg_gmg_plan* plan, int* cycles, double* relres, int* status, long long* total_cycles,
                 void* stream);
/* Counters since sg_gmg_bind (synchronises stream): solves started, cycles run, and
 * solves that ended without reaching tol (cycle cap or non-finite residual). */
int sg_gmg_counters(sg_gmg_plan* plan, long long* solves, long long* cycles, long long* failures, void* stream);
/* sg_gmg_solve_async followed by sg_gmg_stats; returns SG_ERR_NOT_CONVERGED when tol was
 * not reached and SG_ERR_NONFINITE for a NaN/Inf residual. Synchronises stream. */
int sg_gmg_solve(sg_gmg_plan* plan, void* p, int64_t ld_p, const void* div, int64_t ld_div, int div_dtype,
                 double alpha, double tol, int max_cycles, int* cycles_out, double* relres_out, void* stream);
/* Exactly n_cycles cycles (< 128) launched kernel by kernel, no host synchronisation and
 * no graph (capturable by the caller); writes the relative residual before the first and
 * after each cycle into relres_dev[0..n_cycles] (device). */
int sg_gmg_cycles_async(sg_gmg_plan* plan, void* p, int64_t ld_p, const void* div, int64_t ld_div,
                        int div_dtype, double alpha, int n_cycles, double* relres_dev, void* stream);
/* Kernel nodes of the cached solve graph: before the WHILE node and per cycle. */
int sg_gmg_graph_nodes(const sg_gmg_plan* plan, int* prologue_nodes, int* body_nodes);
/* First level run by the single-block kernel (all coarser levels run inside it). */
int sg_gmg_tail_start(const sg_gmg_plan* plan);

/* Shape of one level of the hierarchy (level 0 is the fine grid). */
int sg_gmg_level_shape(const sg_gmg_plan* plan, int level, int* H, int* W);
/* Run `sweeps` smoother sweeps on one level's workspace buffers (whatever they hold);
 * a building block exposed for timing the smoother in isolation. */
int sg_gmg_smooth_async(sg_gmg_plan* plan, int level, int sweeps, void* stream);
/* 1 when the plan's fine level runs the fused register-tiled kernels (open box, large
 * enough to fill the GPU): pre-smoothing + restriction in one launch, post-smoothing +
 * correction of p + next residual in another. */
int sg_gmg_fine_fused(const sg_gmg_plan* plan);
/* How the plan solves its coarsest level exactly: 0 dense pseudo-inverse, 1 cosine transform
 * in one block, 2 cosine transform as four tiled products, 3 cosine transform as two launches
 * streaming their operands into shared memory with bulk asynchronous copies (when the
 * level's rows are whole 16-byte units), 4 the same on clusters of four CTAs that split every
 * product (when each CTA's share of the stream fits in its shared memory); -1 for a NULL
 * plan. No counterpart in the reference. */
int sg_gmg_coarse_solve_kind(const sg_gmg_plan* plan);
/* Timing hook for kernel-by-kernel solves (the fixed-cycle entry points; never inside stream
 * capture): events[2k] and events[2k + 1] (cudaEvent_t, created by the caller with timing
 * enabled) are recorded on the solve's stream right before and after the k-th fused
 * fine-level post launch that follows this call, for k < n_pairs; n_pairs = 0 clears it. The
 * plan keeps the handles, not the events. For timing the solver's dominant kernel in the
 * context of a real step. No counterpart in the reference. */
int sg_gmg_set_post_events(sg_gmg_plan* plan, void* const* events, int n_pairs);
/* One launch of a fused fine-level kernel on the bound workspace, whatever it holds
 * (which = 0: pre kernel; 1: post kernel, which adds its correction to p, ld_p >= W, in the
 * plan's fine precision). Exposed for timing the solver's dominant kernels in isolation;
 * the solve itself runs them inside its graph. No counterpart in the reference. */
int sg_gmg_fine_kernel_async(sg_gmg_plan* plan, int which, void* p, int64_t ld_p, void* stream);

/* ---------------------------------------------------------------- host read-back
 * Device copy of `rows` rows of `row_bytes` bytes (strides in bytes) into a staging buffer,
 * with cache-streaming loads and stores so that the copy does not evict the solver's working
 * set from L2; for reading a field back to the host while the simulation keeps stepping (the
 * reference's get_density_field, common/simulation.py:322-324, returns the live array).
 * Pointers, strides and row_bytes must be multiples of 16 bytes. */
int sg_stage_copy(int64_t rows, int64_t row_bytes, const void* src, int64_t ld_src_bytes, void* dst,
                  int64_t ld_dst_bytes, void* stream);

/* ---------------------------------------------------------------- adjoint (gradients)
 * Reverse-mode kernels of the smoke step with a per-step control force, for gradients of a
 * loss on the final state; the reference has no differentiation, so none of these has a
 * counterpart there. Fields have the MAC shapes of the forward operators; every lam_* output
 * is ACCUMULATED (+=) unless stated, so the caller zeroes it first. */

/* Forward control: u[j][i] += dt fu[j][i] (i < W), v[j][i] += dt fv[j][i] (j < H); fu, fv
 * are H x W. */
int sg_add_control(int dtype, int64_t H, int64_t W, void* u, int64_t ld_u, void* v, int64_t ld_v, const void* fu,
                   int64_t ld_fu, const void* fv, int64_t ld_fv, double dt, void* stream);

/* Workspace bytes of sg_adjoint_advect_scalar (gather = 1: the deterministic form). */
int64_t sg_adjoint_advect_scalar_workspace(int dtype, int64_t H, int64_t W, int gather);
/* Adjoint of sg_advect_scalar (cell-centred field advected by (u, v), then x dissipation):
 * lam_src += transpose(interpolation) lam_out (gather = 0: atomicAdd scatter; 1:
 * deterministic gather over the stored backtrace stencils), and lam_u / lam_v += the
 * velocity part. `src` is the field that was advected. */
int sg_adjoint_advect_scalar(int dtype, int64_t H, int64_t W, const void* lam_out, int64_t ld_lo, const void* src,
                             int64_t ld_src, const void* u, int64_t ld_u, const void* v, int64_t ld_v, int mask_mode,
                             const uint8_t* is_fluid, int64_t ld_fluid, double dt, double cell_size,
                             double dissipation, void* lam_src, int64_t ld_ls, void* lam_u, int64_t ld_lu, void* lam_v,
                             int64_t ld_lv, int gather, void* workspace, int64_t workspace_bytes, void* stream);
/* Adjoint of sg_advect_velocity: (lam_u, lam_v) += adjoint w.r.t. the old (u, v) of the
 * advected faces' adjoints (lam_u_new, lam_v_new); atomicAdd scatter. */
int sg_adjoint_advect_velocity(int dtype, int64_t H, int64_t W, const void* lam_u_new, int64_t ld_lun,
                               const void* lam_v_new, int64_t ld_lvn, const void* u, int64_t ld_u, const void* v,
                               int64_t ld_v, int mask_mode, const uint8_t* fmu, int64_t ld_fmu, const uint8_t* fmv,
                               int64_t ld_fmv, double dt, double cell_size, void* lam_u, int64_t ld_lu, void* lam_v,
                               int64_t ld_lv, void* stream);
/* Adjoint of the density buoyancy term of sg_apply_forces (lam_d += ...) and of
 * sg_add_control (grad_fu = dt lam_u[:, :W], grad_fv = dt lam_v[:H, :], written, either may
 * be NULL). */
int sg_adjoint_forces(int dtype, int64_t H, int64_t W, const void* lam_u, int64_t ld_lu, const void* lam_v,
                      int64_t ld_lv, void* lam_d, int64_t ld_ld, void* grad_fu, int64_t ld_gu, void* grad_fv,
                      int64_t ld_gv, double dt, double gravity, double density_coefficient, void* stream);
/* Adjoint of sg_project: lam_u_out / lam_v_out = the identity part (written), lam_p =
 * -s G^T lam (written), s = dt / (rho h). The pressure's adjoint then goes through the same
 * Poisson solve (lam_div = solve(lam_p)) and sg_adjoint_divergence. */
int sg_adjoint_project(int dtype, int64_t H, int64_t W, const void* lam_u, int64_t ld_lu, const void* lam_v,
                       int64_t ld_lv, void* lam_u_out, int64_t ld_lou, void* lam_v_out, int64_t ld_lov, void* lam_p,
                       int64_t ld_lp, int mask_mode, const uint8_t* fmu, int64_t ld_fmu, const uint8_t* fmv,
                       int64_t ld_fmv, int solid_mode, const uint8_t* solid, int64_t ld_s, double fluid_density,
                       double cell_size, double dt, void* stream);
/* Adjoint of sg_compute_divergence: (lam_u, lam_v) += D^T lam_div. */
int sg_adjoint_divergence(int dtype, int64_t H, int64_t W, const void* lam_div, int64_t ld_ld, void* lam_u,
                          int64_t ld_lu, void* lam_v, int64_t ld_lv, int mask_mode, const uint8_t* fmu, int64_t ld_fmu,
                          const uint8_t* fmv, int64_t ld_fmv, double cell_size, void* stream);

/* ---------------------------------------------------------------- batched scenes
 * Many independent default scenes (open box, solid ring, one overwriting plume, float32)
 * of uneven sizes stepped together: one persistent launch per operator over a tile work
 * list, the multigrid solve to a per-scene relative-residual tolerance, the whole step
 * captured in a CUDA graph. The reference steps one scene per SmokeSimulation2D; these
 * entries have no counterpart there. */
typedef struct sg_batch sg_batch;

/* n_scenes scenes of H[s] x W[s] cells; params: 10 doubles per scene (cell size, dt,
 * fluid density, gravity, density buoyancy coefficient, plume cx, cy, radius (cells),
 * plume density, plume v). Host only. */
int sg_batch_create(sg_batch** out, int n_scenes, const int* H, const int* W, const double* params, double tol,
                    int max_cycles, uint64_t seed);
void sg_batch_destroy(sg_batch* batch);
/* Device workspace the batch needs (fields, hierarchy, work lists, state). */
int64_t sg_batch_workspace_bytes(const sg_batch* batch);
/* Bind a zero-filled state in `workspace` (256-byte aligned) and build the step graphs. */
int sg_batch_bind(sg_batch* batch, void* workspace, int64_t bytes, void* stream);
/* Tile shape (index into sg_batch_tile_shape), smoother sweeps per side, cycle 0 V / 1 W. */
int sg_batch_configure(sg_batch* batch, int tile, int sweeps, int wcycle);
int sg_batch_tile_shape(int tile, int* tx, int* ty);
/* Advance every scene by n_steps steps (graph launches on `stream`). */
int sg_batch_step(sg_batch* batch, int n_steps, void* stream);
/* Byte offsets into the workspace of scene s's current density (H x W), u (H x (W+1)),
 * v ((H+1) x W) and pressure (H x W), float32, row stride = row length. */
int sg_batch_layout(const sg_batch* batch, int scene, int64_t* off_density, int64_t* off_u, int64_t* off_v,
                    int64_t* off_pressure);
/* Which of the two density buffers holds the current state (0 / 1); the velocity state
 * always lives in the first velocity buffer (the projection writes it back there). */
int sg_batch_current(const sg_batch* batch);
/* Cycle-loop iterations (one per cycle of all scenes together) since bind; synchronises. */
int sg_batch_loops(sg_batch* batch, long long* loops, void* stream);
int sg_batch_graph_nodes(const sg_batch* batch, int* step_nodes, int* cycle_nodes);
/* Per-scene outcome of the last solve (host arrays, any may be NULL); synchronises. */
int sg_batch_stats(sg_batch* batch, int* cycles, double* relres, long long* total_cycles, void* stream);
/* Scratch bytes the autotuner needs for its snapshot of the state. */
int64_t sg_batch_snapshot_bytes(const sg_batch* batch);
/* Time `steps` steps of every (tile, sweeps in 1..3, V/W) candidate from the current state
 * (restored each time), configure the fastest whose scenes all converged. */
int sg_batch_autotune(sg_batch* batch, int steps, void* scratch, int64_t scratch_bytes, void* stream, int* tile,
                      int* sweeps, int* wcycle, double* ms_per_step);

/* ---------------------------------------------------------------- profiling metrics
 * Replaces the numpy reductions of MetricsRecorder.process (src/cfd/profiling/metrics.py:
 * 113-133) over the scopes of _build_scope_mask (metrics.py:7-29) with the reducers of
 * profiling/config.py:270-299: one launch reduces an H x W field (float32 or float64, row
 * stride ld) in float64 and writes 18 doubles to device memory at `out`, ordered scope
 * (all, interior = [1:-1, 1:-1], boundary = the rest) x reducer (rms, mean, mean_abs, max,
 * max_abs, std with ddof 0). An empty scope gives NaN. `workspace`:
 * sg_field_stats_workspace_bytes() bytes of device memory, 256-byte aligned, zero-filled
 * before first use; launches sharing one workspace must be stream-ordered. */
int64_t sg_field_stats_workspace_bytes(void);
int sg_field_stats(int dtype, int64_t H, int64_t W, const void* field, int64_t ld, void* workspace, double* out,
                   void* stream);

#ifdef __cplusplus
}
#endif

#endif /* SMOKE_B200_H */
