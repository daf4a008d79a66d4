"""Scene generators: deterministic lattices of cell centres, as the reference's
`block%cell_center` builds them (m_particles.f90:460-479: x outer loop, y
inner loop, centres at (i-1)*dx + dx/2), zone-tagged into real and virtual
particles the way the `input_*.f90` generators do (input_tank.f90,
input_soilfail.f90, input_mix_Savage.f90).  Real particles come first, then
virtual (boundary) particles, each in lattice order (take_real /
take_virtual, m_particles.f90:808-893).

The sizes follow the workloads this library is measured on:
  dam_break()        water column 0.2 x 0.4 in a 0.8 x 0.6 tank, dx 0.005 (4,008 particles)
  granular_column()  soil column 0.2 x 0.1 in a 1.0 x 0.3 box, dx 0.002 (6,608)
  two_phase()        4.0 x 1.0 domain, soil block 1.0 x 0.4, water to 0.8 m, dx 0.002 (912,016)
Every generator takes its lengths and spacing as arguments, so the parity
tests run the same scenes at small sizes.

Choices stated here because the reference takes them from a case file:
  * water b = rho0*c0^2/gamma, c0 = 10*sqrt(2*9.81*H) (the reference reads b
    and c separately, declarations_sph.f90:290);
  * water viscosity 1.0e-3 Pa s;
  * soil K = E/(3(1-2nu)), c = sqrt((K + 4G/3)/rho0), G = E/(2(1+nu));
  * initial soil stress from K0 = 1 - sin(phi): with P the vertical
    overburden, p = (1+2K0)/3 P, sxx = (1-K0)/3 P, syy = -2(1-K0)/3 P.  The
    reference's fixed split 0.1905/-0.381/0.619 (input_soilfail.f90:61-66)
    is this formula at K0 = 0.4285;
  * hsml = dx*1.2 with 1.2 a single-precision literal (input_mix_Savage.f90:60).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from .abi import (SPHG_FP32, SPHG_FP64, SPHG_SOIL, SPHG_WATER, Params, PhaseArrays,
                  default_params, f32)

H_FACTOR = f32(1.2)


@dataclass
class Scene:
    name: str
    params: Params
    phases: list = field(default_factory=list)   # [PhaseArrays] (1 or 2)
    box: tuple = (0.0, 0.0, 0.0)                  # (left wall, right wall, floor)

    @property
    def n_particles(self) -> int:
        return sum(p.n for p in self.phases)

    def copy(self) -> "Scene":
        return Scene(self.name, _copy_params(self.params), [p.copy() for p in self.phases], self.box)


def _copy_params(p: Params) -> Params:
    q = Params()
    import ctypes
    ctypes.memmove(ctypes.addressof(q), ctypes.addressof(p), ctypes.sizeof(Params))
    return q


def lattice(x0: float, y0: float, m: int, n: int, dx: float):
    """Cell centres of an m x n block at (x0, y0), x outer / y inner."""
    i = np.repeat(np.arange(m), n)
    j = np.tile(np.arange(n), m)
    x = i * dx + dx / 2.0 + x0
    y = j * dx + dx / 2.0 + y0
    return x, y


def _phase(x, y, real_mask, virt_mask, material, dx):
    xr, yr = x[real_mask], y[real_mask]
    xv, yv = x[virt_mask], y[virt_mask]
    n = xr.size + xv.size
    P = PhaseArrays(n, xr.size, material, dspp=dx)
    P.x[:, 0] = np.concatenate([xr, xv])
    P.x[:, 1] = np.concatenate([yr, yv])
    P.hsml[:] = dx * H_FACTOR
    sign = 2 if material == SPHG_WATER else 3   # setup_itype m_particles.f90:896-913
    P.itype[:xr.size] = sign
    P.itype[xr.size:] = -sign
    return P


def _box(width, height, dx, layers=2):
    """Lattice covering a width x height box plus `layers` virtual rows under
    the floor and columns outside both walls."""
    m = int(round(width / dx)) + 2 * layers
    n = int(round(height / dx)) + layers
    x, y = lattice(-layers * dx, -layers * dx, m, n, dx)
    virt = (x < 0.0) | (x > width) | (y < 0.0)
    return x, y, virt


def _water_material(depth, rho0=1000.0, gamma=7.0, mu=1.0e-3):
    c0 = 10.0 * math.sqrt(2.0 * 9.81 * depth)
    return dict(rho0=rho0, gamma=gamma, c=c0, b=rho0 * c0 * c0 / gamma, viscosity=mu)


def _soil_material(rho0=1850.0, E=0.84e6, nu=0.3, phi_deg=19.8, cohesion=0.0,
                   porosity=0.4, permeability=1.0e-3):
    K = E / (3.0 * (1.0 - 2.0 * nu))
    G = E / (2.0 * (1.0 + nu))
    c = math.sqrt((K + 4.0 * G / 3.0) / rho0)
    return dict(rho0=rho0, E=E, niu=nu, k=K, G=G, c=c, phi=math.radians(phi_deg),
                cohesion=cohesion, porosity=porosity, permeability=permeability)


def _set_material(mat, d):
    for k, v in d.items():
        setattr(mat, k, v)


def _k0_stress(P: PhaseArrays, overburden: np.ndarray, phi: float):
    k0 = 1.0 - math.sin(phi)
    P.p[:] = (1.0 + 2.0 * k0) / 3.0 * overburden
    P.sxx[:] = (1.0 - k0) / 3.0 * overburden
    P.syy[:] = -2.0 * (1.0 - k0) / 3.0 * overburden
    P.sxy[:] = 0.0


def _initial_density(P: PhaseArrays, wm: dict):
    """initial_density, m_particles.f90:2105-2130 (inverse Tait)."""
    P.rho[:] = wm["rho0"] * (P.p / wm["b"] + 1.0) ** (1.0 / wm["gamma"])


def _finish(p: Params, phases, width, height, dx, skf, precision):
    p.skf = skf
    p.precision = precision
    margin = 8 * dx
    p.x_min, p.x_max = -2 * dx - margin, width + 2 * dx + margin
    p.y_min, p.y_max = -2 * dx - margin, 2.0 * height + margin
    # capacity of each pair list: ~12 pairs per particle at support 2h, scaled
    # with the support area for the 3h kernels
    sk = 3 if skf in (2, 3) else 2
    p.max_interaction = int(3 * sk * sk * max(ph.n for ph in phases)) + 4096


def dam_break(width=0.2, height=0.4, tank_w=0.8, tank_h=0.6, dx=0.005, skf=1,
              precision=SPHG_FP64) -> Scene:
    """Water dam-break (water-only step, declarations_sph.f90:1439)."""
    x, y, virt = _box(tank_w, tank_h, dx)
    real = (~virt) & (x < width) & (y < height)
    P = _phase(x, y, real, virt, SPHG_WATER, dx)
    p = default_params()
    wm = _water_material(height)
    _set_material(p.water, wm)
    g = p.gravity
    yy, xx = P.x[:, 1], P.x[:, 0]
    P.p[:] = wm["rho0"] * g * (yy - height)
    P.p[P.ntotal:][(xx[P.ntotal:] >= width) | (yy[P.ntotal:] > height)] = 0.0
    P.c[:] = wm["c"]
    P.vof[:] = 1.0
    _initial_density(P, wm)
    P.mass[:] = dx * dx * P.rho
    p.single_phase = 1
    p.first_material = SPHG_WATER
    p.alpha, p.beta, p.delta = 0.1, 0.0, 0.1
    p.dt = 0.25 * float(P.hsml[0]) / wm["c"]
    _finish(p, [P], tank_w, tank_h, dx, skf, precision)
    return Scene("dam_break", p, [P], (0.0, tank_w, 0.0))


def granular_column(width=0.2, height=0.1, box_w=1.0, box_h=0.3, dx=0.002, skf=1,
                    phi_deg=19.8, precision=SPHG_FP32) -> Scene:
    """Dry granular column collapse (soil-only step, declarations_sph.f90:1530)."""
    x, y, virt = _box(box_w, box_h, dx)
    real = (~virt) & (x < width) & (y < height)
    P = _phase(x, y, real, virt, SPHG_SOIL, dx)
    p = default_params()
    sm = _soil_material(phi_deg=phi_deg)
    _set_material(p.soil, sm)
    g = p.gravity
    xx, yy = P.x[:, 0], P.x[:, 1]
    over = np.maximum(sm["rho0"] * g * (yy - height), 0.0)
    over[P.ntotal:][xx[P.ntotal:] >= width] = 0.0
    _k0_stress(P, over, sm["phi"])
    P.c[:] = sm["c"]
    P.rho[:] = sm["rho0"]
    P.mass[:] = dx * dx * P.rho
    p.single_phase = 1
    p.first_material = SPHG_SOIL
    p.alpha = 0.1
    p.dt = 0.1 * float(P.hsml[0]) / sm["c"]
    _finish(p, [P], box_w, box_h, dx, skf, precision)
    return Scene("granular_column", p, [P], (0.0, box_w, 0.0))


def two_phase(width=4.0, height=1.0, block_w=1.0, block_h=0.4, water_h=0.8, dx=0.002,
              porosity=0.4, permeability=1.0e-3, skf=1, phi_deg=19.8, precision=SPHG_FP32,
              forchheimer_b=0.0) -> Scene:
    """Submerged soil block under a water layer (two-phase step,
    declarations_sph.f90:1131), laid out as input_mix_Savage.f90 does: the
    water lattice fills the block too, as the pore-water phase.
    forchheimer_b [s^2/m^2] > 0 adds the quadratic Forchheimer drag to the
    reference's linear Darcy law (0: the reference's law)."""
    x, y, virt = _box(width, height, dx)
    inside = ~virt
    in_block = (x < block_w) & (y < block_h)
    W = _phase(x, y, inside & (y < water_h), virt, SPHG_WATER, dx)
    S = _phase(x, y, inside & in_block, virt, SPHG_SOIL, dx)
    p = default_params()
    wm = _water_material(water_h)
    sm = _soil_material(porosity=porosity, permeability=permeability, phi_deg=phi_deg)
    _set_material(p.water, wm)
    _set_material(p.soil, sm)
    g = p.gravity
    # water: hydrostatic pressure, porosity inside the block
    wx, wy = W.x[:, 0], W.x[:, 1]
    W.p[:] = np.maximum(wm["rho0"] * g * (wy - water_h), 0.0)
    W.c[:] = wm["c"]
    W.vof[:] = 1.0
    W.vof[(wx < block_w) & (wy < block_h)] = porosity
    _initial_density(W, wm)
    W.rho *= W.vof
    W.mass[:] = dx * dx * W.rho
    # soil: buoyant overburden, K0 stress, solid fraction 1 - porosity
    sx, sy = S.x[:, 0], S.x[:, 1]
    over = np.maximum((sm["rho0"] - wm["rho0"]) * g * (sy - block_h), 0.0)
    over[S.ntotal:][(sx[S.ntotal:] >= block_w) | (sy[S.ntotal:] >= block_h)] = 0.0
    _k0_stress(S, over, sm["phi"])
    S.c[:] = sm["c"]
    S.vof[:] = 1.0 - porosity
    S.rho[:] = sm["rho0"] * S.vof
    S.mass[:] = dx * dx * S.rho
    p.single_phase = 0
    p.alpha = 0.1
    p.forchheimer_b = forchheimer_b
    h = float(W.hsml[0])
    p.dt = min(0.25 * h / wm["c"], 0.1 * h / sm["c"])
    _finish(p, [W, S], width, height, dx, skf, precision)
    return Scene("two_phase", p, [W, S], (0.0, width, 0.0))


def jitter(scene: Scene, amplitude: float, seed: int = 12345) -> Scene:
    """Displace real particles by U(-a, a) per axis (breaks lattice ties)."""
    s = scene.copy()
    rng = np.random.default_rng(seed)
    for P in s.phases:
        P.x[:P.ntotal] += rng.uniform(-amplitude, amplitude, size=(P.ntotal, 2))
    return s


def small(name: str, precision=None, skf=1) -> Scene:
    """Reduced-size versions of the three workloads, for parity tests."""
    if name == "dam_break":
        return dam_break(width=0.05, height=0.1, tank_w=0.2, tank_h=0.15, dx=0.005, skf=skf,
                         precision=SPHG_FP64 if precision is None else precision)
    if name == "granular_column":
        return granular_column(width=0.04, height=0.02, box_w=0.12, box_h=0.05, dx=0.002, skf=skf,
                               precision=SPHG_FP32 if precision is None else precision)
    if name == "two_phase":
        return two_phase(width=0.2, height=0.1, block_w=0.05, block_h=0.03, water_h=0.06, dx=0.002,
                         skf=skf, precision=SPHG_FP32 if precision is None else precision)
    raise ValueError(name)
