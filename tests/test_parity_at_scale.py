"""Parity at the benchmark configurations' own sizes: the engine (FP64 and
mixed forms, through the C ABI) against the FP64 oracle on the host.

  C2  inverse-stiffness beam, 12,800 tets, all 60 steps, forward + adjoint
  C3  muscle star refined twice (9,840 tets) on the ground, 20 steps (one
      checkpoint segment of 20), dL/dE and dL/dactivation
  C4  64 x 64 cloth on the ball, 10 steps through its first contacts (from
      the oracle's state 26 steps after the drop), dL/dx0 and dL/dv0.  Longer
      windows cannot hold 1e-9: once contact passes accumulate, the scheme
      amplifies a rounding-level difference about tenfold per step (measured:
      1e-14 after 1 step, 1e-9 after 16, 1e-2 after 28, with every contact
      pass and iteration count still equal, and with the GPU's four execution
      paths — fused or looped contact phase, broad phase or not — agreeing
      bit for bit among themselves)
  C5  8 scenes of the 256-scene uneven batch, evenly spaced in size (1,035 to
      49,010 tets), as one batch, 100 steps, dL/dE and dL/dactivation

Tolerances: FP64 positions and velocities 1e-9 relative to the oracle's
scale, gradients 1e-8; mixed positions 1e-6, velocities 1e-6 in position
units (|dv| h against the largest position), gradients 1e-4; iteration
counts and contact passes equal in FP64.
"""
import dataclasses
import os

import numpy as np
import pytest

from diff_fem_b200 import _capi, scene as S
from diff_fem_b200.engine import Scene
from oracle import oracle as O

pytestmark = pytest.mark.gpu

THREADS = os.cpu_count() or 1


def rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def oracle_run(d, x, v, n, act, seed):
    o = O.OracleScene(d)
    ro = o.forward(x, v, n_steps=n, act=act, traj=True, threads=THREADS)
    rng = np.random.default_rng(seed)
    gx, gv = rng.standard_normal(x.size), rng.standard_normal(x.size)
    bo = o.backward(gx, gv)
    return o, ro, bo, gx, gv


def gpu_run(g, x, v, n, act, gx, gv):
    xg, vg, tg = g.forward(x, v, n_steps=n, act=act, traj=True)
    return xg, vg, tg, g.backward(gx, gv)


def check(d, n, keys, act=None, x=None, v=None, seed=0, mixed=True):
    x = d.x0.reshape(-1).copy() if x is None else x
    v = np.zeros_like(x) if v is None else v
    o, ro, bo, gx, gv = oracle_run(d, x, v, n, act, seed)
    errs = {}
    g = Scene(d)
    xg, vg, tg, bg = gpu_run(g, x, v, n, act, gx, gv)
    assert np.array_equal(g.iterations(n), ro["iters"])
    assert np.array_equal(g.contact_passes(n), o.contact_passes())
    errs["fp64"] = {"traj": rel(tg, ro["traj"]), "v": rel(vg, ro["v"]), **{k: rel(bg[k], bo[k]) for k in keys}}
    g.close()
    assert errs["fp64"]["traj"] < 1e-9 and errs["fp64"]["v"] < 1e-9, errs
    for k in keys:
        assert errs["fp64"][k] < 1e-8, (k, errs)
    if mixed:
        gm = Scene(dataclasses.replace(d, precision=_capi.DFEM_PREC_MIXED))
        xm, vm, tm, bm = gpu_run(gm, x, v, n, act, gx, gv)
        scale = np.abs(ro["x"]).max()
        errs["mixed"] = {"traj": rel(tm, ro["traj"]), "v_pos_units": float(np.abs(vm - ro["v"]).max() * d.time_step / scale),
                         **{k: rel(bm[k], bo[k]) for k in keys}}
        gm.close()
        assert errs["mixed"]["traj"] < 1e-6 and errs["mixed"]["v_pos_units"] < 1e-6, errs
        for k in keys:
            assert errs["mixed"][k] < 1e-4, (k, errs)
    return errs


def test_c2_inverse_stiffness_all_60_steps():
    check(S.inverse_stiffness(), 60, ("x", "v", "E", "nu"))


def test_c3_muscle_star_on_the_ground_one_checkpoint_segment():
    d = dataclasses.replace(S.muscle_star(refine=2), checkpoint_every=20)
    act = np.random.default_rng(42).uniform(0, 1, (20, d.n_segments))
    errs = check(d, 20, ("x", "v", "E", "act"), act=act)
    assert errs is not None


def test_c4_cloth_on_the_ball_through_its_first_contacts():
    d = S.cloth_on_ball()
    x0 = d.x0.reshape(-1).copy()
    r = O.OracleScene(d).forward(x0, np.zeros_like(x0), n_steps=26, threads=THREADS)
    check(d, 10, ("x", "v"), x=r["x"], v=r["v"])


def test_c5_sample_of_the_uneven_batch_as_one_batch():
    """8 scenes of the batch workload, evenly spaced in size, stepped as one
    batch handle in both forms against the oracle scene by scene (the stars
    without their ground: over 100 steps contact passes amplify rounding, as
    in the C4 window; batches with contact are checked bit for bit against
    the scenes alone in tests/test_batch.py)."""
    descs, _ = S.uneven_batch(n_scenes=256, precision=_capi.DFEM_PREC_FP64, ground=False)
    order = np.argsort([q.n_tets for q in descs], kind="stable")
    pick = [descs[i] for i in order[np.linspace(0, len(descs) - 1, 8).astype(int)]]
    n = 100
    rng = np.random.default_rng(7)
    acts = [rng.uniform(0, 1, (n, q.n_segments)) if q.n_segments else None for q in pick]
    ref = []
    for q, a in zip(pick, acts):
        x = q.x0.reshape(-1).copy()
        ref.append(oracle_run(q, x, np.zeros_like(x), n, a, seed=len(ref)))
    x = np.concatenate([q.x0.reshape(-1) for q in pick])
    act = np.concatenate([a for a in acts if a is not None], axis=1)
    gx = np.concatenate([r[3] for r in ref])
    gv = np.concatenate([r[4] for r in ref])
    for prec in (_capi.DFEM_PREC_FP64, _capi.DFEM_PREC_MIXED):
        b = Scene.batch([dataclasses.replace(q, precision=prec) for q in pick])
        xb, vb, tb, bb = gpu_run(b, x, np.zeros_like(x), n, act, gx, gv)
        vo, to, so = b.offsets["vertices"], b.offsets["tets"], b.offsets["segments"]
        tb = tb.reshape(n, -1)
        it = b.iterations(n)
        for p, (o, ro, bo, _, _) in enumerate(ref):
            a0, a1 = 3 * vo[p], 3 * vo[p + 1]
            ep = rel(tb[:, a0:a1], ro["traj"].reshape(n, -1))
            eE = rel(bb["E"][to[p]:to[p + 1]], bo["E"])
            ea = rel(bb["act"][:, so[p]:so[p + 1]], bo["act"]) if so[p + 1] > so[p] else 0.0
            if prec == _capi.DFEM_PREC_FP64:
                assert np.array_equal(it[:, p], ro["iters"]), p
                assert ep < 1e-9 and eE < 1e-8 and ea < 1e-8, (p, ep, eE, ea)
            else:
                assert ep < 1e-6 and eE < 1e-4 and ea < 1e-4, (p, ep, eE, ea)
        b.close()
