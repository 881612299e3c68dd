"""Oracle: CPU restatement of bfps' Lagrangian tracer step.

TEST INFRASTRUCTURE ONLY (the checker for the CUDA gather + Adams-Bashforth
kernel); the product never imports it.

Follows, single-rank semantics:

* particles_system::completeLoop (bfps/cpp/particles/particles_system.hpp:210-217):
  compute rhs[0] = u(x) -> move (AB of order min(step_idx, nsteps)) ->
  redistribute -> step_idx += 1 -> rotate the rhs history and zero rhs[0].
* particles_field_computer::get_norm_pos_in_cell / pbc_field_layer /
  apply_computation (particles_field_computer.hpp:55-63, 65-157, 176-183):
  the (2n+2)^3 tensor-product gather, summed z-outer, x-middle, y-inner,
  with coefficient (bz*by)*bx and the field value promoted to double.
* particles_adams_bashforth::move_particles (particles_adams_bashforth.hpp:18-133).
* the box is [0, 2*pi/dk) per axis with spacing box/N
  (particles_system_builder.hpp:176-191).

Redistribution on one rank only reorders the arrays by z-layer
(particles_distr_mpi.hpp:798-831); outputs are written in global index order
(particles_output_hdf5.hpp), so the oracle keeps particles in index order.
"""
import math
import numpy as np

from .interp import beta_eval

MAX_AB_STEPS = 6


def ab_update(pos, rhs, order, dt):
    """particles_adams_bashforth.hpp:41-131, same expression forms."""
    if order > MAX_AB_STEPS:
        raise RuntimeError("Step in particles_adams_bashforth is too large")
    r = rhs
    if order == 1:
        return pos + dt * r[0]
    if order == 2:
        return pos + dt * (3. * r[0] - r[1]) / 2.
    if order == 3:
        return pos + dt * (23. * r[0] - 16. * r[1] + 5. * r[2]) / 12.
    if order == 4:
        return pos + dt * (55. * r[0] - 59. * r[1] + 37. * r[2] - 9. * r[3]) / 24.
    if order == 5:
        return pos + dt * (1901. * r[0] - 2774. * r[1] + 2616. * r[2] - 1274. * r[3]
                           + 251. * r[4]) / 720.
    if order == 6:
        return pos + dt * (4277. * r[0] - 7923. * r[1] + 9982. * r[2] - 7298. * r[3]
                           + 2877. * r[4] - 475. * r[5]) / 1440.
    return pos


class Geometry:
    def __init__(self, nx, ny, nz, dkx=1.0, dky=1.0, dkz=1.0):
        self.grid = (nx, ny, nz)
        # 4 * acos(0) / dk (particles_system_builder.hpp:176-179)
        self.box = tuple(4 * math.acos(0) / d for d in (dkx, dky, dkz))
        self.step = tuple(self.box[i] / float(self.grid[i]) for i in range(3))

    def norm_pos_in_cell(self, pos, d):
        L = self.box[d]
        h = self.step[d]
        nb = np.floor(pos / L)
        pib = pos - nb * L
        cell = np.floor(pib / h)
        return (pib - cell * h) / h

    def field_layer(self, pos, d):
        lvl = np.floor(pos / self.step[d]).astype(np.int64)
        n = self.grid[d]
        return np.mod(lvl, n)


def sample(field_r, pos, n, m, geom):
    """apply_computation for a real field (nz, ny, nx, ncomp) at positions (P, 3).

    Returns (P, ncomp) float64, accumulated in the reference order.
    """
    nx, ny, nz = geom.grid
    ncomp = field_r.shape[-1]
    px, py, pz = pos[:, 0], pos[:, 1], pos[:, 2]
    bx = beta_eval(n, m, geom.norm_pos_in_cell(px, 0))
    by = beta_eval(n, m, geom.norm_pos_in_cell(py, 1))
    bz = beta_eval(n, m, geom.norm_pos_in_cell(pz, 2))
    gx = geom.field_layer(px, 0)
    gy = geom.field_layer(py, 1)
    gz = geom.field_layer(pz, 2)
    out = np.zeros((pos.shape[0], ncomp))
    f = field_r
    for iz in range(2 * n + 2):
        z = np.mod(gz - n + iz, nz)
        for ix in range(2 * n + 2):
            x = np.mod(gx - n + ix, nx)
            for iy in range(2 * n + 2):
                y = np.mod(gy - n + iy, ny)
                coef = (bz[iz] * by[iy]) * bx[ix]
                vals = f[z, y, x].astype(np.float64)
                out += vals * coef[:, None]
    return out


class ParticlesSystem:
    """Single-rank ``particles_system`` in global index order."""

    def __init__(self, pos, rhs, neighbours, smoothness, geom, step_idx=1):
        self.pos = np.array(pos, dtype=np.float64, copy=True)
        self.rhs = np.array(rhs, dtype=np.float64, copy=True)  # (nsteps, P, 3)
        self.n = neighbours
        self.m = smoothness
        self.geom = geom
        self.step_idx = step_idx

    @property
    def nsteps(self):
        return self.rhs.shape[0]

    def complete_loop(self, field_r, dt):
        # compute(): rhs[0] += u(x) (rhs[0] is zero after the previous shift)
        self.rhs[0] = self.rhs[0] + sample(field_r, self.pos, self.n, self.m, self.geom)
        # move()
        order = min(self.step_idx, self.nsteps)
        self.pos = ab_update(self.pos, self.rhs, order, dt)
        # redistribute(): reorder only (no effect in index order)
        self.step_idx += 1
        # shift_rhs_vectors()
        if self.nsteps:
            self.rhs = np.roll(self.rhs, 1, axis=0)
            self.rhs[0] = 0
