"""Per-phase device times of one PD iteration (dfem_profile_phases): the
local step, the gather, the global solve and the adjoint local step, each
launched outside the step graphs so that a profiler sees them one by one.

    python -m diff_fem_b200.phases --workload c2|batch32 [--precision fp64|mixed]
                                   [--solve auto|levels|persistent|split|cluster|resident] [--reps 5]

c2: the inverse-stiffness beam (12,800 tets); batch32: 32 scenes of the
uneven batch (beams and muscle stars, without their grounds) as one handle.
"""
from __future__ import annotations

import argparse

import numpy as np


def main(argv=None) -> dict:
    p = argparse.ArgumentParser()
    p.add_argument("--workload", default="c2", choices=["c2", "batch32"])
    p.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    p.add_argument("--solve", default=None)
    p.add_argument("--reps", type=int, default=5)
    a = p.parse_args(argv)
    import torch
    from . import scene as S
    from ._capi import DFEM_PREC_FP64, DFEM_PREC_MIXED
    from .engine import Scene
    prec = DFEM_PREC_MIXED if a.precision == "mixed" else DFEM_PREC_FP64
    if a.workload == "c2":
        d = S.inverse_stiffness(precision=prec)
        sc = Scene(d)
        x = torch.tensor(d.x0.reshape(-1), device="cuda")
        act = None
    else:
        descs, _ = S.uneven_batch(n_scenes=32, precision=prec, ground=False)
        sc = Scene.batch(descs)
        x = torch.tensor(np.concatenate([q.x0.reshape(-1) for q in descs]), device="cuda")
        act = torch.tensor(np.random.default_rng(1).uniform(0, 1, (1, sc.nseg)), device="cuda")
    if a.solve:
        print(sc.solve_mode(a.solve))
    sc.forward(x, torch.zeros_like(x), n_steps=1, act=act)
    ms = sc.profile_phases(reps=a.reps)
    print({"workload": a.workload, "precision": a.precision, "solve": sc.solve_mode()["mode"], "ms": ms})
    return ms


if __name__ == "__main__":
    main()
