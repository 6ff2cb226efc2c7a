"""Mixed form (FP32 projections and slot accumulation, FP64 state, rhs,
factor and solves) against the FP64 oracle.

Tolerances of the mixed form: positions 1e-6 relative to the largest
position magnitude; velocities 1e-6 in position units (|dv| h against the
largest position magnitude: the near-static scenes have velocities close to 0,
so a tolerance relative to max |v| would measure round-off of a difference);
gradients 1e-4 relative to each gradient's largest magnitude.
"""
import numpy as np
import pytest

from diff_fem_b200 import _capi, scene as S
from diff_fem_b200.engine import Scene
from oracle import oracle as O

pytestmark = pytest.mark.gpu

POS_TOL = 1e-6
GRAD_TOL = 1e-4


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def check(d64, dmx, n, act=None, x=None, keys=("x", "v", "E", "nu"), seed=0):
    x = d64.x0.reshape(-1).copy() if x is None else x
    v = np.zeros_like(x)
    o = O.OracleScene(d64)
    ro = o.forward(x, v, n_steps=n, act=act, traj=True)
    g = Scene(dmx)
    xg, vg, tg = g.forward(x, v, n_steps=n, act=act, traj=True)
    g64 = Scene(d64)
    x64, _ = g64.forward(x, v, n_steps=n, act=act)
    g64.close()
    assert not np.array_equal(xg, x64)  # the mixed kernels ran
    assert rel(tg, ro["traj"]) < POS_TOL
    assert np.abs(vg - ro["v"]).max() * d64.time_step < POS_TOL * np.abs(ro["x"]).max()
    rng = np.random.default_rng(seed)
    gx, gv = rng.standard_normal(x.size), rng.standard_normal(x.size)
    bg, bo = g.backward(gx, gv), o.backward(gx, gv)
    errs = {k: rel(bg[k], bo[k]) for k in keys}
    for k, e in errs.items():
        assert e < GRAD_TOL, (k, e)
    g.close()
    return errs


def test_inverse_stiffness_mixed():
    kw = dict(nx=16, ny=4, nz=4)
    check(S.inverse_stiffness(**kw), S.inverse_stiffness(precision=_capi.DFEM_PREC_MIXED, **kw), 4)


def test_muscles_mixed():
    n = 5
    d64, dmx = S.muscle_beam(), S.muscle_beam(precision=_capi.DFEM_PREC_MIXED)
    act = np.random.default_rng(2).uniform(0, 1, (n, d64.n_segments))
    check(d64, dmx, n, act=act, keys=("x", "v", "E", "nu", "act"))


def test_cloth_mixed():
    d64 = S.cloth_sheet(nv=10)
    dmx = S.cloth_sheet(nv=10, precision=_capi.DFEM_PREC_MIXED)
    check(d64, dmx, 6, keys=("x", "v"))


def test_flattened_elements_take_the_fp64_branch():
    """Every element starts with a smallest / largest singular value near 0.03
    (the body squashed along y), below the FP32 branch's threshold."""
    kw = dict(nx=8, ny=3, nz=3)
    d64 = S.inverse_stiffness(**kw)
    dmx = S.inverse_stiffness(precision=_capi.DFEM_PREC_MIXED, **kw)
    x = d64.x0.reshape(-1, 3).copy()
    x[:, 1] = x[:, 1].mean() + 0.03 * (x[:, 1] - x[:, 1].mean())
    check(d64, dmx, 3, x=x.reshape(-1))
