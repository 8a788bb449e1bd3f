"""FP64 PyTorch-autodiff restatement of the controlled smoke step (test infrastructure).

Same operations as adjoint.ControlledSmoke.forward_step on the default scene (open-box
kernel masks, solid ring for the boundary zeroing, exact float64 buoyancy), written with
plain torch ops so that torch.autograd differentiates it: overwriting plume discs, buoyancy
(forces.py:19-46 face averaging), control on the left / lower faces, semi-Lagrangian
advection with the reference's clamped bilinear sample (advection.py:6-49, 97-180),
dissipation, divergence (divergence.py:4-25), an exact pressure solve (pseudo-inverse of the
Neumann Laplacian; it differs from an iterative solve only by a constant, which the
projection ignores) and the projection (pressure_gradient.py:4-37, boundaries.py:7-39).
Only for small grids.
"""
import torch


def sample(f, x, y):
    rows, cols = f.shape
    x0 = torch.floor(x).clamp(0, cols - 1)
    x1 = torch.ceil(x).clamp(0, cols - 1)
    y0 = torch.floor(y).clamp(0, rows - 1)
    y1 = torch.ceil(y).clamp(0, rows - 1)
    tx, ty = x - x0, y - y0
    x0, x1, y0, y1 = (a.long() for a in (x0, x1, y0, y1))
    c00, c10, c01, c11 = f[y0, x0], f[y0, x1], f[y1, x0], f[y1, x1]
    c0 = c00 + (c10 - c00) * tx
    c1 = c01 + (c11 - c01) * tx
    return c0 + (c1 - c0) * ty


class RefStep:
    def __init__(self, H, W, h, dt, gravity, plumes, dissipation=0.999, rho=1.0, dc=1.0):
        self.H, self.W, self.h, self.dt, self.g = H, W, h, dt, gravity
        self.plumes = [list(map(float, r)) for r in plumes]
        self.diss, self.rho, self.dc = dissipation, rho, dc
        d = torch.float64
        j, i = torch.meshgrid(torch.arange(H, dtype=d), torch.arange(W + 1, dtype=d), indexing="ij")
        self.uj, self.ui = j, i
        j, i = torch.meshgrid(torch.arange(H + 1, dtype=d), torch.arange(W, dtype=d), indexing="ij")
        self.vj, self.vi = j, i
        j, i = torch.meshgrid(torch.arange(H, dtype=d), torch.arange(W, dtype=d), indexing="ij")
        self.cj, self.ci = j, i
        # open-box face masks
        self.mu = ((self.ui >= 1) & (self.ui <= W - 1)).to(d)
        self.mv = ((self.vj >= 1) & (self.vj <= H - 1)).to(d)
        # faces the projection keeps (open and not next to a ring cell)
        self.ou = ((self.ui >= 2) & (self.ui <= W - 2) & (self.uj >= 1) & (self.uj <= H - 2)).to(d)
        self.ov = ((self.vj >= 2) & (self.vj <= H - 2) & (self.vi >= 1) & (self.vi <= W - 2)).to(d)
        # Neumann Laplacian over all cells (open box) and its pseudo-inverse
        n = H * W
        A = torch.zeros((n, n), dtype=d)
        for jj in range(H):
            for ii in range(W):
                c = jj * W + ii
                for dj, di in ((0, -1), (0, 1), (-1, 0), (1, 0)):
                    a, b = jj + dj, ii + di
                    if 0 <= a < H and 0 <= b < W:
                        A[c, c] += 1.0
                        A[c, a * W + b] -= 1.0
        self.Ainv = torch.linalg.pinv(A)
        self.alpha = -h * h * rho / dt

    def __call__(self, d, u, v, fu, fv):
        H, W, h, dt = self.H, self.W, self.h, self.dt
        for cx, cy, r, dval, vval, _noise in self.plumes:
            r2 = r * r
            inside = (self.ci + 0.5 - cx) ** 2 + (self.cj + 0.5 - cy) ** 2 < r2
            d = torch.where(inside, torch.full_like(d, dval), d)
            inside = (self.vi + 0.5 - cx) ** 2 + (self.vj - cy) ** 2 < r2
            v = torch.where(inside, torch.full_like(v, vval), v)
            inside = (self.ui - cx) ** 2 + (self.uj + 0.5 - cy) ** 2 < r2
            u = torch.where(inside, torch.zeros_like(u), u)
        # buoyancy: face j takes d[j] at j = 0 and H - 1, the mean of d[j - 1], d[j] between
        rows = [d[0:1]]                                   # face 0: d[0]
        if H > 2:
            rows.append(0.5 * (d[0:H - 2] + d[1:H - 1]))  # faces 1 .. H-2: (d[j-1] + d[j]) / 2
        if H > 1:
            rows.append(d[H - 1:H])                       # face H-1: d[H-1]
        rows.append(torch.zeros((1, W), dtype=d.dtype))   # face H: nothing
        dd = torch.cat(rows, 0)
        v = v + dt * (-self.dc * dd * self.g)
        u = torch.cat([u[:, :W] + dt * fu, u[:, W:]], 1)
        v = torch.cat([v[:H] + dt * fv, v[H:]], 0)
        k = dt / h
        # velocity self-advection
        uu = u
        vv = sample(v, self.ui - 0.5, self.uj + 0.5)
        u2 = sample(u, self.ui - uu * k, self.uj + 0.5 - vv * k - 0.5) * self.mu
        uu = sample(u, self.vi + 0.5, self.vj - 0.5)
        vv = v
        v2 = sample(v, self.vi + 0.5 - uu * k - 0.5, self.vj - vv * k) * self.mv
        # density advection with the advected velocity
        uu = sample(u2, self.ci + 0.5, self.cj)
        vv = sample(v2, self.ci, self.cj + 0.5)
        d2 = self.diss * sample(d, self.ci + 0.5 - uu * k - 0.5, self.cj + 0.5 - vv * k - 0.5)
        # projection
        um, vm = u2 * self.mu, v2 * self.mv
        div = ((um[:, 1:] - um[:, :-1]) + (vm[1:] - vm[:-1])) / h
        p = (self.Ainv @ (self.alpha * div.reshape(-1))).reshape(H, W)
        s = dt / (self.rho * h)
        gu = torch.zeros_like(u2)
        gu[:, 1:W] = p[:, 1:] - p[:, :-1]
        gv = torch.zeros_like(v2)
        gv[1:H] = p[1:] - p[:-1]
        u3 = (u2 - s * gu) * self.ou
        v3 = (v2 - s * gv) * self.ov
        return d2, u3, v3
