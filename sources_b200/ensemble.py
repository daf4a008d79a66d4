"""Batched ensembles: many independent scenes stepped together.

The reference's program holds one scene.  An ensemble groups its scenes by
step kind (water-only dam-breaks, dry soil collapses, submerged two-phase
collapses), places the scenes of a group side by side along x with gaps
wider than the kernel support, and uploads each group as ONE libsphg
context: every kernel of a step then processes every scene of the group in
the same launch, and each step of a group is one CUDA-graph replay.  The
parameters that differ between scenes (time step, water b and c from the
water depth, soil friction angle) live in the per-scene table of the
context (sphg_set_scenes), indexed by a per-particle scene id.

Scene parameters come from a counter-based generator: Philox4x32-10 keyed
by the scene seed (numpy.random.Philox(key=seed)), so scene s is the same
whatever the ensemble size.  Ranges (per scene): kind uniform over the three
step kinds; real particles of the column log-uniform in [2,000, 60,000];
column aspect H/W uniform in [0.5, 4]; friction angle uniform in [20, 40]
degrees; water depth uniform in [0.1, 0.5] m (the water level above the
soil of a submerged scene); spacing dx = 0.004 m.

An autotuner picks the neighbour-cell factor, the reorder interval and the
number of x cells per neighbour cell of each group by timing a few steps of
every candidate on a throw-away copy of the group.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from . import Solver, SolverGroup, scenes
from .abi import SPHG_FP32, SPHG_SOIL, SPHG_WATER, Params, PhaseArrays
from .scenes import Scene, _copy_params

KINDS = ("dam_break", "dry", "submerged")


@dataclass
class SceneSpec:
    seed: int
    kind: str
    n_target: int       # real particles of the column
    aspect: float       # column height / width
    phi_deg: float
    depth: float        # water above the soil (submerged scenes)


def spec(seed: int) -> SceneSpec:
    g = np.random.Generator(np.random.Philox(key=seed))
    u = g.random(5)
    kind = KINDS[min(int(u[0] * 3), 2)]
    n = int(round(math.exp(math.log(2000) + u[1] * (math.log(60000) - math.log(2000)))))
    return SceneSpec(seed, kind, n, 0.5 + 3.5 * u[2], 20.0 + 20.0 * u[3], 0.1 + 0.4 * u[4])


def specs(n_scenes: int, first_seed: int = 0):
    return [spec(first_seed + s) for s in range(n_scenes)]


def _column(sp: SceneSpec, n: int, dx: float):
    w = dx * math.sqrt(n / sp.aspect)
    h = sp.aspect * w
    w = max(round(w / dx), 2) * dx
    h = max(round(h / dx), 2) * dx
    return w, h


def build_scene(sp: SceneSpec, dx: float = 0.004, precision=SPHG_FP32, skf: int = 1) -> Scene:
    """One scene of the ensemble, in its own coordinates."""
    if sp.kind == "dam_break":
        w, h = _column(sp, sp.n_target, dx)
        tank_w = round(max(4.0 * w, w + 0.4) / dx) * dx
        return scenes.dam_break(width=w, height=h, tank_w=tank_w, tank_h=round(1.2 * h / dx) * dx, dx=dx,
                                skf=skf, precision=precision)
    if sp.kind == "dry":
        w, h = _column(sp, sp.n_target, dx)
        box_w = round(max(w + 3.0 * h, w + 0.3) / dx) * dx
        return scenes.granular_column(width=w, height=h, box_w=box_w, box_h=round(1.2 * h / dx) * dx, dx=dx,
                                      skf=skf, phi_deg=sp.phi_deg, precision=precision)
    # submerged: the soil column holds a third of the target, water fills the box to h + depth
    w, h = _column(sp, max(sp.n_target // 3, 200), dx)
    water_h = round((h + sp.depth) / dx) * dx
    box_w = round(max(w + 2.0 * h, 2.0 * w) / dx) * dx
    return scenes.two_phase(width=box_w, height=round(1.2 * water_h / dx) * dx, block_w=w, block_h=h,
                            water_h=water_h, dx=dx, skf=skf, phi_deg=sp.phi_deg, precision=precision)


def scene_row(s: Scene):
    p = s.params
    return (p.dt, p.water.b, p.water.c, p.soil.phi)


@dataclass
class Group:
    kind: str
    scene: Scene                 # the packed scene
    members: list                # indices into the ensemble's scene list
    ranges: list                 # per phase: [(start, stop) of each member]
    offsets: list                # x offset of each member
    rows: list                   # per-scene table rows
    sids: list                   # per phase: scene id of every particle
    tuning: tuple = (1.0, 10, 0)


def pack(members, built, gap_cells: float = 6.0) -> Group:
    """Place the scenes of one kind side by side along x."""
    first = built[members[0]]
    nph = len(first.phases)
    h = max(float(b.phases[0].hsml.max()) for b in (built[m] for m in members))
    gap = gap_cells * 3.0 * h      # several support radii between neighbouring scenes
    cursor = 0.0
    parts = [[] for _ in range(nph)]
    ranges = [[] for _ in range(nph)]
    sids = [[] for _ in range(nph)]
    offsets, rows = [], []
    counts = [0] * nph
    y_min, y_max = math.inf, -math.inf
    cap = 0
    for local, m in enumerate(members):
        s = built[m]
        off = cursor - s.params.x_min
        offsets.append(off)
        rows.append(scene_row(s))
        for k, P in enumerate(s.phases):
            Q = P.copy()
            Q.x[:, 0] += off
            parts[k].append(Q)
            ranges[k].append((counts[k], counts[k] + P.n))
            counts[k] += P.n
            sids[k].append(np.full(P.n, local, dtype=np.int32))
        cursor = s.params.x_max + off + gap
        y_min = min(y_min, s.params.y_min)
        y_max = max(y_max, s.params.y_max)
        cap += s.params.max_interaction
    packed = []
    for k in range(nph):
        n = counts[k]
        nt = sum(Q.ntotal for Q in parts[k])
        R = PhaseArrays(n, nt, parts[k][0].material, parts[k][0].dspp)
        for f in ("x", "vx", "rho", "p", "c", "mass", "hsml", "vof", "sxx", "sxy", "syy", "itype"):
            getattr(R, f)[...] = np.concatenate([getattr(Q, f) for Q in parts[k]])
        packed.append(R)
    prm = _copy_params(first.params)
    prm.x_min, prm.x_max = 0.0, cursor
    prm.y_min, prm.y_max = y_min, y_max
    prm.max_interaction = cap
    prm.dt = min(r[0] for r in rows)
    return Group(first.name, Scene(first.name + "_batch", prm, packed), list(members), ranges, offsets, rows,
                 [np.concatenate(x) for x in sids])


def _solver(g: Group, tuning):
    sv = Solver(g.scene)
    sv.set_scenes(g.rows)
    for k, ids in enumerate(g.sids):
        sv.upload_scene_ids(k + 1, ids)
    sv.set_tuning(*tuning)
    return sv


# (cell factor, reorder interval, x cells per cell)
CANDIDATES = [(1.0, 10, 4), (1.0, 25, 4), (1.0, 10, 2), (1.0, 10, 1), (1.25, 10, 4), (1.25, 25, 4), (1.5, 10, 4)]


def autotune(g: Group, steps: int = 8, warmup: int = 3, candidates=CANDIDATES):
    """Time every (cell factor, reorder interval, x split) candidate on a
    copy of the group and return the fastest with the table of timings
    (ms/step)."""
    table = {}
    for cand in candidates:
        sv = _solver(g, cand)
        sv.time_integration(warmup)
        sv.time_integration(steps)
        table[cand] = sv.stats().last_step_ms
        sv.close()
    best = min(table, key=table.get)
    return best, table


class Ensemble:
    def __init__(self, spec_list, dx: float = 0.004, precision=SPHG_FP32, skf: int = 1, tune: bool = True):
        self.specs = list(spec_list)
        self.built = [build_scene(sp, dx=dx, precision=precision, skf=skf) for sp in self.specs]
        self.groups = []
        self.tuning_table = {}
        for kind in KINDS:
            members = [i for i, sp in enumerate(self.specs) if sp.kind == kind]
            if not members:
                continue
            g = pack(members, self.built)
            g.kind = kind
            if tune:
                g.tuning, self.tuning_table[kind] = autotune(g)
            self.groups.append(g)
        self.solvers = [_solver(g, g.tuning) for g in self.groups]
        self.group = None

    @property
    def n_particles(self) -> int:
        return sum(g.scene.n_particles for g in self.groups)

    def set_stream(self, handle):
        for sv in self.solvers:
            sv.set_stream(handle)

    def time_integration(self, nsteps: int):
        """Every group nsteps steps: one CUDA graph per step for all groups
        (SolverGroup) once they are built."""
        if self.group is None:
            self.group = SolverGroup(self.solvers)
        self.group.time_integration(nsteps)

    def scene(self, index: int):
        """Per-phase PhaseArrays of one scene, in its own coordinates."""
        for g, sv in zip(self.groups, self.solvers):
            if index in g.members:
                local = g.members.index(index)
                out = []
                for k in range(len(g.scene.phases)):
                    full = sv.download(k + 1)
                    a, b = g.ranges[k][local]
                    P = self.built[index].phases[k]
                    Q = PhaseArrays(P.n, P.ntotal, P.material, P.dspp)
                    for f in ("x", "vx", "dvx", "av", "rho", "drho", "p", "c", "vof", "dvof", "sxx", "sxy", "syy",
                              "dsxx", "dsxy", "dsyy", "dp", "itype", "fail"):
                        getattr(Q, f)[...] = getattr(full, f)[a:b]
                    Q.x[:, 0] -= g.offsets[local]
                    out.append(Q)
                return out
        raise IndexError(index)

    def close(self):
        if self.group is not None:
            self.group.close()
            self.group = None
        for sv in self.solvers:
            sv.close()
        self.solvers = []
