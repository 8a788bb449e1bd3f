"""SmokeSimulation2D on CUDA: the reference simulator's API over the CUDA kernels.

Mirrors src/cfd/common/simulation.py:19-335: constructor ``(config, profiler=None)``,
the same attributes (density, velocity_u, velocity_v, pressure, temperature,
divergence, pressure_residual, is_fluid, _face_mask_u/_v, _solid_mask, dt, gravity,
buoyancy, ...), the same phase order in ``substep`` and the accumulator ``update``.
Fields are torch CUDA tensors (float32 like the reference, or float64).

Reference behaviour kept on purpose:
  * the face masks are built from an all-fluid solid mask before the 1-cell solid
    ring is painted (simulation.py:102-113 then :126-131), so until set_solid_mask()
    the solve sees every interior face open and the ring only acts through
    enforce_boundary_conditions;
  * the solve uses ``self.dt`` while the other phases use the ``dt`` argument
    (simulation.py:311-312);
  * pressure restarts from zero every step (:310) and the metrics tail (divergence
    and residual after projection, :251-265) always runs.

Exact fusions (results unchanged): the density dissipation is applied inside the
density advection (nothing reads density in between); gradient subtraction and
boundary enforcement run in one pass; the two velocity advections run in one launch.
The temperature chain (advect, cool, temperature force) is skipped while the
temperature field is provably ambient everywhere: no temperature emitter has fired,
the field was never handed out, and ambient_temperature is 0 -- in which case the
reference computes exact zeros for it.
"""
from __future__ import annotations

import contextlib

import numpy as np
import torch

from . import _lib as L
from . import operators as ops
from .operators import OPEN_BOX, RING_BOX
from .params import DEFAULT_SOLVER_PARAMS
from .solvers import calculate_alpha, calculate_reciprocal_beta, solve_pressure


class _NullTiming:
    enabled = False

    @contextlib.contextmanager
    def scope(self, name):
        yield


class _NullMetrics:
    enabled = False

    def capture(self, *args, **kwargs):
        pass

    def process(self):
        pass

    def tick(self, frame):
        pass


class NullProfileSession:
    """Disabled profiling session with the reference's interface (profiling/session.py:12-55)."""

    def __init__(self):
        self.timing = _NullTiming()
        self.metrics = _NullMetrics()
        self._frame = 0

    @property
    def enabled(self):
        return False

    def tick(self):
        self._frame += 1

    def reset(self):
        pass


APPROACHES = ("linear", "gaussian", "quadratic", "hard_cutoff")


class Emitter2D:
    """Additive emitter with the reference's constructor and accessors (common/emitters.py:69-208).

    ``emit`` adds value * falloff(dist) * dt inside the radius to each non-zero
    channel (emitters.py:202-221), with dist measured from the integer cell index.
    ``numba_optimized`` is accepted for compatibility; both reference paths compute
    the same values (the CUDA kernel follows the Numba path's arithmetic).
    """

    def __init__(self, position, radius, density_value=1.0, temperature_value=0.0, velocity_value=(0.0, 0.0),
                 approach="linear", numba_optimized=False):
        if approach not in APPROACHES:
            raise ValueError(f"Unknown emission approach: {approach}")
        self.position = position
        self.radius = radius
        self.approach = approach
        self.density_value = density_value
        self.temperature_value = temperature_value
        self.velocity_value = velocity_value
        self.enabled = True
        self.numba_optimized = numba_optimized

    def emit(self, density_field, velocity_u_field, velocity_v_field, temperature_field, dt):
        emit_channels(self, density_field, velocity_u_field, velocity_v_field, temperature_field, dt)

    def set_enabled(self, enabled):
        self.enabled = enabled

    def set_position(self, position):
        self.position = position

    def set_radius(self, radius):
        self.radius = radius

    def set_density_value(self, v):
        self.density_value = v

    def set_temperature_value(self, v):
        self.temperature_value = v

    def set_velocity_value(self, v):
        self.velocity_value = v

    def to_dict(self):
        return {"position": self.position, "radius": self.radius, "density_value": self.density_value,
                "temperature_value": self.temperature_value, "velocity_value": self.velocity_value,
                "approach": self.approach, "numba_optimized": self.numba_optimized}

    @classmethod
    def from_dict(cls, data):
        return cls(position=data.get("position", (0, 0)), radius=data.get("radius", 5.0),
                   density_value=data.get("density_value", 1.0), temperature_value=data.get("temperature_value", 0.0),
                   velocity_value=data.get("velocity_value", (0.0, 0.0)), approach=data.get("approach", "linear"),
                   numba_optimized=data.get("numba_optimized", False))


def emit_channels(e, density, u, v, temperature, dt):
    """emitters.py:202-221 for any emitter-like object (this package's or the reference's)."""
    if not getattr(e, "enabled", True):
        return
    px, py = e.position
    r = e.radius
    a = e.approach
    if density is not None and e.density_value != 0.0:
        ops.emit_scalar(density, e.density_value, dt, px, py, r, a)
    if temperature is not None and e.temperature_value != 0.0:
        ops.emit_scalar(temperature, e.temperature_value, dt, px, py, r, a)
    if u is not None and e.velocity_value[0] != 0.0:
        ops.emit_scalar(u, e.velocity_value[0], dt, px, py, r, a)
    if v is not None and e.velocity_value[1] != 0.0:
        ops.emit_scalar(v, e.velocity_value[1], dt, px, py, r, a)


class PlumeSource:
    """Overwriting disc source of the benchmark scenes (no reference counterpart).

    Each step, cells whose centre (i+.5, j+.5) lies strictly inside the disc get
    ``density_value``; v faces at (i+.5, j) get ``v_value`` plus uniform noise in
    [-noise_amp, noise_amp); u faces at (i, j+.5) get the noise alone. The noise is a
    counter hash of (seed, step, component, row, column). Coordinates are in cells.
    """

    def __init__(self, cx, cy, radius, density_value=1.0, v_value=1.0, noise_amp=0.0):
        self.cx, self.cy, self.radius = float(cx), float(cy), float(radius)
        self.density_value, self.v_value, self.noise_amp = float(density_value), float(v_value), float(noise_amp)

    def row(self):
        return [self.cx, self.cy, self.radius, self.density_value, self.v_value, self.noise_amp]


class SmokeSimulation2D:
    """Real-time 2-D smoke simulator (semi-Lagrangian advection + pressure projection) on CUDA."""

    def __init__(self, config, profiler=None, *, device=None, dtype=torch.float32, seed: int = 0):
        self.config = config
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.dtype = dtype
        self.seed = seed
        self._initialise_from_config(config, profiler)

    # ------------------------------------------------------------ construction
    def _initialise_from_config(self, config, profiler):
        self.width, self.height = config.grid.size
        self.cell_size = config.grid.cell_size
        self.pressure_solver_method = config.pressure_solver.method
        # this simulator runs the CUDA registrations whatever backend the config names
        self.pressure_solver_backend = "cuda"
        params = config.pressure_solver.params
        self.solver_params = params if params is not None else DEFAULT_SOLVER_PARAMS[self.pressure_solver_method]
        self.operators_backend = config.operators
        self.domain_width = self.width * self.cell_size
        self.domain_height = self.height * self.cell_size
        self.dt = 0.016
        self.accumulator = 0.0
        self.max_substeps = 4
        self.density_dissipation = 0.999
        self.buoyancy = 5.0
        self.gravity = -0.5
        self.fluid_density = 1.0
        H, W = self.height, self.width
        z = lambda *s: torch.zeros(s, dtype=self.dtype, device=self.device)  # noqa: E731
        self.density, self.density_temp = z(H, W), z(H, W)
        self.velocity_u, self.velocity_u_temp = z(H, W + 1), z(H, W + 1)
        self.velocity_v, self.velocity_v_temp = z(H + 1, W), z(H + 1, W)
        self.pressure = z(H, W)
        self._temperature, self.temperature_temp = z(H, W), z(H, W)
        self.ambient_temperature = 0.0
        self.cooling_rate = 0.5
        self.divergence = z(H, W)
        self.pressure_residual = z(H, W)
        self._temperature_active = False
        # simulation.py:101-113: masks from an all-fluid solid mask, then the ring (:126-131)
        self._face_mask_u, self._face_mask_v, self.is_fluid = ops.build_masks(
            torch.zeros((H, W), dtype=torch.bool, device=self.device))
        self._solid_mask = torch.zeros((H, W), dtype=torch.bool, device=self.device)
        self._init_boundaries()
        self._kmasks = (OPEN_BOX, OPEN_BOX, OPEN_BOX)  # kernels evaluate the open-box masks
        self._ksolid = RING_BOX
        self._mask_dirty = False
        self.emitters = []
        self.plumes = []
        self._plume_table = None
        self.step_index = 0
        self.debug = getattr(config, "debug", False)
        self.profiler = profiler if profiler is not None else NullProfileSession()
        # "reference": the reference's float64 sampling arithmetic, bit for bit; "float32":
        # float32 fields advected in float32 arithmetic (equal up to rounding, faster)
        self.advection_arithmetic = "reference"
        # forces and the projection tail (projection, divergence and residual after it):
        # "reference" (float64 terms, bit for bit) or, for float32 fields, "float32"
        self.operator_arithmetic = "reference"

    def _init_boundaries(self):
        self._solid_mask[0, :] = True
        self._solid_mask[-1, :] = True
        self._solid_mask[:, 0] = True
        self._solid_mask[:, -1] = True

    # ------------------------------------------------------------ temperature field
    @property
    def temperature(self):
        """The temperature field; handing it out re-enables the temperature chain."""
        self._temperature_active = True
        return self._temperature

    @temperature.setter
    def temperature(self, t):
        self._temperature_active = True
        self._temperature = t

    def _temperature_needed(self):
        if self.ambient_temperature != 0.0:
            self._temperature_active = True
        if any(getattr(e, "enabled", True) and e.temperature_value != 0.0 for e in self.emitters):
            self._temperature_active = True
        return self._temperature_active

    # ------------------------------------------------------------ masks
    def set_solid_mask(self, solid_mask):
        """simulation.py:133-143; masks are rebuilt at the next substep."""
        t = torch.as_tensor(solid_mask, device=self.device)
        if tuple(t.shape) != (self.height, self.width):
            raise ValueError(f"Solid mask must have shape ({self.height}, {self.width})")
        self._solid_mask = t.bool().contiguous()
        self._mask_dirty = True

    def get_solid_mask(self):
        return self._solid_mask.clone()

    def _rebuild_masks(self):
        self._face_mask_u, self._face_mask_v, self.is_fluid = ops.build_masks(self._solid_mask)
        self._kmasks = (self._face_mask_u, self._face_mask_v, self.is_fluid)
        self._ksolid = self._solid_mask
        self._mask_dirty = False

    # ------------------------------------------------------------ sources
    def add_emitter(self, emitter):
        self.emitters.append(emitter)

    def add_plume(self, plume: PlumeSource):
        self.plumes.append(plume)
        self._plume_table = None

    def set_plumes(self, plumes):
        self.plumes = list(plumes)
        self._plume_table = None

    def set_plume_table(self, table):
        """Use a caller-owned (n, 6) float64 HOST table of plume rows (cx, cy, r, density,
        v, noise), e.g. refreshed by the caller every step; it is read at each substep and
        travels to the GPU in the launch parameters."""
        self._plume_table = table

    # ------------------------------------------------------------ stepping
    def update(self, frame_dt):
        """simulation.py:166-184: fixed substeps with an accumulator and a spiral-of-death clamp."""
        self.accumulator += frame_dt
        substeps = 0
        while self.accumulator >= self.dt and substeps < self.max_substeps:
            self.substep(self.dt)
            self.accumulator -= self.dt
            substeps += 1
        if substeps >= self.max_substeps:
            self.accumulator = 0.0

    def substep(self, dt):
        """One substep in the reference's order (simulation.py:186-265)."""
        prof = self.profiler
        prof.tick()
        if self._mask_dirty:
            self._rebuild_masks()
        scope = prof.timing.scope
        with scope("simulation.substep"):
            with scope("simulation.emitters"):
                self._apply_emitters(dt)
            with scope("simulation.forces"):
                self._apply_forces(dt)
            with scope("simulation.advection.velocity"):
                self._advect_velocity(dt)
            with scope("simulation.advection.density"):
                self._advect_density(dt)
            temp_on = self._temperature_active
            with scope("simulation.advection.temperature"):
                if temp_on:
                    self._advect_temperature(dt)
            with scope("simulation.cooling"):
                if temp_on:
                    self._cool_temperature(dt)
            with scope("simulation.dissipation"):
                pass  # applied inside the density advection
            with scope("simulation.divergence"):
                self._compute_divergence()
            with scope("profiling.capture"):
                prof.metrics.capture("divergence", "before_projection", self.divergence)
            with scope("simulation.pressure.solve"):
                self._solve_pressure()
            with scope("simulation.pressure.apply"):
                # projection plus the metrics tail's divergence and residual in one pass
                self._project_and_metrics(dt)
        with scope("profiling.metrics"):
            prof.metrics.capture("divergence", "after_projection", self.divergence)
            prof.metrics.capture("pressure", "final", self.pressure)
            prof.metrics.capture("pressure_residual", "final", self.pressure_residual)
            prof.metrics.process()
        self.step_index += 1

    def _apply_emitters(self, dt):
        temp = self._temperature if self._temperature_needed() else None
        for e in self.emitters:
            emit_channels(e, self.density, self.velocity_u, self.velocity_v, temp, dt)
        if self.plumes or self._plume_table is not None:
            if self._plume_table is None:
                self._plume_table = np.asarray([p.row() for p in self.plumes], dtype=np.float64).reshape(-1, 6)
            ops.plume_sources(self.density, self.velocity_u, self.velocity_v, self._plume_table, self.seed,
                              self.step_index)

    def _apply_forces(self, dt):
        temp = self._temperature if self._temperature_active else None
        ops.apply_forces(self.velocity_v, self.density, temp, dt, self.gravity, self.buoyancy, 1.0,
                         self.ambient_temperature, arithmetic=self.operator_arithmetic)

    def _advect_velocity(self, dt):
        fmu, fmv, _ = self._kmasks
        ops.advect_velocity(self.velocity_u, self.velocity_u_temp, self.velocity_v, self.velocity_v_temp, fmu, fmv, dt,
                            self.cell_size, arithmetic=self.advection_arithmetic)
        self.velocity_u, self.velocity_u_temp = self.velocity_u_temp, self.velocity_u
        self.velocity_v, self.velocity_v_temp = self.velocity_v_temp, self.velocity_v

    def _advect_density(self, dt):
        _, _, fl = self._kmasks
        ops.advect_scalar_field(self.density, self.density_temp, self.velocity_u, self.velocity_v, fl, dt,
                                self.cell_size, dissipation=self.density_dissipation,
                                arithmetic=self.advection_arithmetic)
        self.density, self.density_temp = self.density_temp, self.density

    def _advect_temperature(self, dt):
        _, _, fl = self._kmasks
        ops.advect_scalar_field(self._temperature, self.temperature_temp, self.velocity_u, self.velocity_v, fl, dt,
                                self.cell_size, arithmetic=self.advection_arithmetic)
        self._temperature, self.temperature_temp = self.temperature_temp, self._temperature

    def _compute_divergence(self):
        fmu, fmv, _ = self._kmasks
        ops.compute_divergence(self.velocity_u, self.velocity_v, self.divergence, fmu, fmv, self.cell_size)

    def _cool_temperature(self, dt):
        ops.cool_temperature(self._temperature, self.ambient_temperature, self.cooling_rate, dt)

    def _solve_pressure(self):
        fmu, fmv, _ = self._kmasks
        # simulation.py:310 zeroes the pressure before every solve; the multigrid solve from a
        # zero guess does not read it (it writes p = 0 itself), so the fill is skipped there
        if not (self.pressure_solver_method == "geometric_multigrid"
                and not getattr(self.solver_params, "fixed_cycles", 0)):
            self.pressure.zero_()
        solve_pressure(self.pressure, self.divergence, fmu, fmv, self.fluid_density, self.cell_size, self.dt, self,
                       zero_initial_guess=True)

    def _apply_pressure_gradient(self, dt):
        fmu, fmv, _ = self._kmasks
        ops.apply_pressure_gradient(self.velocity_u, self.velocity_v, self.pressure, fmu, fmv, self.fluid_density,
                                    self.cell_size, dt)

    def _enforce_boundaries(self):
        ops.enforce_boundary_conditions(self.velocity_u, self.velocity_v, self._ksolid)

    def _project_and_metrics(self, dt):
        """simulation.py:244-265 fused: the projected velocity (written to the spare buffers,
        then swapped in), the divergence after projection and the pressure residual."""
        fmu, fmv, fl = self._kmasks
        ops.project_metrics(self.velocity_u, self.velocity_v, self.velocity_u_temp, self.velocity_v_temp,
                            self.pressure, fmu, fmv, fl, self._ksolid, self.fluid_density, self.cell_size, dt,
                            calculate_alpha(self.cell_size, self.fluid_density, dt), calculate_reciprocal_beta(),
                            self.divergence, self.pressure_residual, arithmetic=self.operator_arithmetic)
        self.velocity_u, self.velocity_u_temp = self.velocity_u_temp, self.velocity_u
        self.velocity_v, self.velocity_v_temp = self.velocity_v_temp, self.velocity_v

    def _project(self, dt):
        fmu, fmv, _ = self._kmasks
        ops.project(self.velocity_u, self.velocity_v, self.pressure, fmu, fmv, self._ksolid, self.fluid_density,
                    self.cell_size, dt)

    # ------------------------------------------------------------ accessors
    def get_density_field(self):
        return self.density

    def reset(self):
        for t in (self.density, self.velocity_u, self.velocity_v, self._temperature, self.pressure, self.divergence):
            t.zero_()
        self.accumulator = 0.0


class FieldReadback:
    """Host read-back of a simulation field every step without stalling the steps.

    ``SmokeSimulation2D.get_density_field`` (common/simulation.py:322-324) hands out the live
    array; on the GPU the next substep rewrites it in place (the sources) while a host copy
    would still be reading it. ``submit()``, called after a substep, copies the field on the
    device into one of ``slots`` staging buffers (cache-streaming loads and stores,
    sg_stage_copy) and queues its copy into pinned host memory on a copy stream; a slot is
    reused only after its previous host copy has finished (the compute stream waits for it on
    the device, not the host). ``result(slot)`` waits for that slot's copy and returns the
    pinned host tensor."""

    def __init__(self, sim, field="density", slots=2):
        self.sim, self.field = sim, field
        src = getattr(sim, field)
        self.host = [torch.empty(src.shape, dtype=src.dtype).pin_memory() for _ in range(slots)]
        self.staging = [torch.empty_like(src) for _ in range(slots)]
        self.copy_stream = torch.cuda.Stream(device=src.device)
        self.done = [None] * slots
        self.next = 0

    def _stage(self, dst, src):
        es = src.element_size()
        rb = src.shape[1] * es
        if (src.data_ptr() | dst.data_ptr() | src.stride(0) * es | dst.stride(0) * es | rb) % 16 == 0 \
                and src.stride(1) == 1 and dst.stride(1) == 1:
            L.call("sg_stage_copy", src.shape[0], rb, src.data_ptr(), src.stride(0) * es, dst.data_ptr(),
                   dst.stride(0) * es, L.stream_ptr())
        else:
            dst.copy_(src)

    def submit(self):
        """Queue the read-back of the field as it stands; returns the slot it lands in."""
        k = self.next
        self.next = (k + 1) % len(self.host)
        stream = torch.cuda.current_stream()
        if self.done[k] is not None:
            stream.wait_event(self.done[k])
        self._stage(self.staging[k], getattr(self.sim, self.field))
        staged = torch.cuda.Event()
        staged.record(stream)
        self.copy_stream.wait_event(staged)
        with torch.cuda.stream(self.copy_stream):
            self.host[k].copy_(self.staging[k], non_blocking=True)
        ev = torch.cuda.Event()
        ev.record(self.copy_stream)
        self.done[k] = ev
        return k

    def wait(self, stream=None):
        """Make `stream` (default: the current one) wait for every queued read-back."""
        stream = stream or torch.cuda.current_stream()
        for ev in self.done:
            if ev is not None:
                stream.wait_event(ev)

    def result(self, slot):
        """The pinned host copy of slot `slot`, after waiting for it on the host."""
        if self.done[slot] is not None:
            self.done[slot].synchronize()
        return self.host[slot]
