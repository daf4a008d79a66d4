"""Step times of the four single-context workloads on the current GPU.

    python -m sources_b200.workloads

Each workload is stepped through warm-up steps, then three windows of steps
are timed with CUDA events on the context's stream; the best window is
reported as one JSON line per workload:

  two_phase_912k FP32   the 912,016-particle two-phase collapse (FP32 pairs, FP64 state)
  two_phase_912k FP64   the same scene in the FP64 parity mode
  dam_break 4k FP64     water column 0.2 x 0.4 m in a 0.8 x 0.6 m tank, dx 5 mm
  granular_column 6.6k  dry soil column 0.2 x 0.1 m in a 1.0 x 0.3 m box, dx 2 mm (FP32)

    python -m sources_b200.workloads ensemble_fixed_cost

times instead the per-step fixed cost of a batched ensemble: three scenes of
2,000 real particles, one of each kind, stepped as the 256-scene ensemble is
(three groups, one joint CUDA graph per step), whose kernels have almost no
work, so the step time is the graph's launch and dependency overhead.
"""
from __future__ import annotations

import json


def time_scene(scene, warm: int, steps: int, label: str) -> dict:
    import torch
    from . import Solver
    stream = torch.cuda.current_stream()
    with Solver(scene) as g:
        g.set_stream(stream.cuda_stream)
        g.time_integration(warm)
        torch.cuda.synchronize()
        best = 1e9
        for _ in range(3):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            g.time_integration(steps)
            e1.record(stream)
            torch.cuda.synchronize()
            best = min(best, e0.elapsed_time(e1) / steps)
    n = scene.n_particles
    return {"case": label, "particles": n, "ms_per_step": round(best, 5), "particle_steps_per_s": n / (best / 1000)}


def ensemble_fixed_cost(warm: int = 20, steps: int = 200) -> dict:
    import torch
    from . import ensemble
    from .ensemble import SceneSpec
    specs = [SceneSpec(0, "dam_break", 2000, 2.0, 30.0, 0.2), SceneSpec(1, "dry", 2000, 2.0, 30.0, 0.2),
             SceneSpec(2, "submerged", 2000, 2.0, 30.0, 0.2)]
    ens = ensemble.Ensemble(specs, tune=False)
    try:
        stream = torch.cuda.current_stream()
        ens.set_stream(stream.cuda_stream)
        ens.time_integration(warm)
        torch.cuda.synchronize()
        best = 1e9
        for _ in range(3):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            ens.time_integration(steps)
            e1.record(stream)
            torch.cuda.synchronize()
            best = min(best, e0.elapsed_time(e1) / steps)
        return {"case": "ensemble_fixed_cost (3 scenes x 2,000 real particles, 3 groups, one graph per step)",
                "particles": ens.n_particles, "ms_per_step": round(best, 5)}
    finally:
        ens.close()


def main():
    import sys
    if "ensemble_fixed_cost" in sys.argv[1:]:
        print(json.dumps(ensemble_fixed_cost()), flush=True)
        return
    from . import scenes
    from .abi import SPHG_FP32, SPHG_FP64
    for args in ((scenes.two_phase(precision=SPHG_FP64), 10, 50, "two_phase_912k FP64"),
                 (scenes.two_phase(precision=SPHG_FP32), 10, 100, "two_phase_912k FP32"),
                 (scenes.dam_break(), 20, 500, "dam_break 4k FP64"),
                 (scenes.granular_column(), 20, 500, "granular_column 6.6k FP32")):
        print(json.dumps(time_scene(*args)), flush=True)


if __name__ == "__main__":
    main()
