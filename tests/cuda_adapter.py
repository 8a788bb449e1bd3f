"""Adapter exposing the CUDA operators with the reference's numpy signatures.

Each call copies the numpy inputs to the device, runs the CUDA operator through the
package (and so through the C ABI), and writes results back into the caller's numpy
arrays in place -- so the reference's known-answer tests (tests/kats.py) and the
golden comparisons run unchanged against the CUDA path.
"""
import numpy as np
import torch

from conftest import package

sg = package()
ops = sg.operators
solvers = sg.solvers


def dev(a):
    if a is None:
        return None
    t = torch.from_numpy(np.ascontiguousarray(a))
    return t.cuda()


def back(t, a):
    a[...] = t.cpu().numpy()


class CudaOps:
    @staticmethod
    def advect_scalar_field(src, dst, u, v, is_fluid, dt, cell_size):
        d = dev(dst)
        ops.advect_scalar_field(dev(src), d, dev(u), dev(v), dev(is_fluid), dt, cell_size)
        back(d, dst)

    @staticmethod
    def advect_velocity_u(us, ud, v, fmu, dt, cell_size):
        d = dev(ud)
        ops.advect_velocity_u(dev(us), d, dev(v), dev(fmu), dt, cell_size)
        back(d, ud)

    @staticmethod
    def advect_velocity_v(vs, vd, u, fmv, dt, cell_size):
        d = dev(vd)
        ops.advect_velocity_v(dev(vs), d, dev(u), dev(fmv), dt, cell_size)
        back(d, vd)

    @staticmethod
    def apply_forces(v, density, temperature, dt, gravity, bc, dc, amb, f32_temporaries=True):
        d = dev(v)
        ops.apply_forces(d, dev(density), dev(temperature), dt, gravity, bc, dc, amb, f32_temporaries=f32_temporaries)
        back(d, v)

    @staticmethod
    def cool_temperature(t, amb, rate, dt):
        d = dev(t)
        ops.cool_temperature(d, amb, rate, dt)
        back(d, t)

    @staticmethod
    def compute_divergence(u, v, div, fmu, fmv, cell_size):
        d = dev(div)
        ops.compute_divergence(dev(u), dev(v), d, dev(fmu), dev(fmv), cell_size)
        back(d, div)

    @staticmethod
    def compute_residual(p, div, fl, fmu, fmv, alpha, rb, out):
        d = dev(out)
        ops.compute_residual(dev(p), dev(div), dev(fl), dev(fmu), dev(fmv), alpha, rb, d)
        back(d, out)
        return out

    @staticmethod
    def apply_pressure_gradient(u, v, p, fmu, fmv, rho, h, dt):
        du, dv = dev(u), dev(v)
        ops.apply_pressure_gradient(du, dv, dev(p), dev(fmu), dev(fmv), rho, h, dt)
        back(du, u)
        back(dv, v)

    @staticmethod
    def enforce_boundary_conditions(u, v, solid):
        du, dv = dev(u), dev(v)
        ops.enforce_boundary_conditions(du, dv, dev(solid))
        back(du, u)
        back(dv, v)

    @staticmethod
    def jacobi_pressure_solver(p, div, fmu, fmv, rho, h, dt, iterations, **kw):
        d = dev(p)
        solvers.jacobi_pressure_solver(d, dev(div), dev(fmu), dev(fmv), rho, h, dt, iterations)
        back(d, p)

    @staticmethod
    def rb_sor_pressure_solver(p, div, fmu, fmv, rho, h, dt, iterations, omega=0.0, **kw):
        d = dev(p)
        solvers.red_black_sor_gauss_seidel_pressure_solver(d, dev(div), dev(fmu), dev(fmv), rho, h, dt, iterations,
                                                           omega=omega)
        back(d, p)

    @staticmethod
    def gauss_seidel_pressure_solver(p, div, fmu, fmv, rho, h, dt, iterations, **kw):
        d = dev(p)
        solvers.gauss_seidel_pressure_solver(d, dev(div), dev(fmu), dev(fmv), rho, h, dt, iterations)
        back(d, p)
