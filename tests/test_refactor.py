"""Numeric refactorisation on the GPU (dfem_set_materials): the factor the
solves use is recomputed on the device from the new moduli, with the
reference's regularise-and-retry rule applied per part of a batch."""
import dataclasses

import numpy as np
import pytest

from diff_fem_b200 import _capi, scene as S
from diff_fem_b200.engine import Scene
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300)


def test_repeated_material_updates_track_the_oracle():
    d = S.inverse_stiffness(nx=12, ny=4, nz=4)
    g, o = Scene(d), O.OracleScene(d)
    x = d.x0.reshape(-1).copy()
    for seed in (11, 12, 13):
        E = S.log_uniform_moduli(d.n_tets, seed)
        nu = np.random.default_rng(seed).uniform(0.2, 0.45, d.n_tets)
        g.set_materials(E, nu)
        o.set_materials(E, nu)
        xg, vg = g.forward(x, np.zeros_like(x), n_steps=3)
        ro = o.forward(x, np.zeros_like(x), n_steps=3)
        assert rel(xg, ro["x"]) < 1e-9
        assert np.array_equal(g.iterations(3), ro["iters"])
    assert g.info()["factor_regularisation"] == 0.0
    g.close()


def test_invalid_material_is_rejected():
    d = S.inverse_stiffness(nx=6, ny=2, nz=2)
    g = Scene(d)
    nu = np.full(d.n_tets, 0.3)
    nu[3] = -1.5
    with pytest.raises(_capi.DfemError, match="invalid material"):
        g.set_materials(np.asarray(d.youngs), nu)
    g.close()


def test_regularisation_retry_is_per_part():
    descs = [dataclasses.replace(S.inverse_stiffness(nx=6, ny=2, nz=2, seed=s), max_iterations=2) for s in (1, 2)]
    b = Scene.batch(descs)
    to = b.offsets["tets"]
    E = np.concatenate([np.asarray(q.youngs) for q in descs])
    E[to[1]:to[2]] = -1e6  # the second part's Hs is indefinite: its factorisation needs a regularisation
    nu = np.full(E.size, 0.3)
    b.set_materials(E, nu)
    assert b.info()["factor_regularisation"] > 0.0
    x = np.concatenate([q.x0.reshape(-1) for q in descs])
    xb, _ = b.forward(x, np.zeros_like(x), n_steps=1)
    s0 = Scene(descs[0])
    s0.solve_mode("persistent")  # the batch's per-supernode arithmetic (the dense form agrees to rounding only)
    s0.set_materials(E[:to[1]], nu[:to[1]])
    x0, _ = s0.forward(descs[0].x0.reshape(-1), np.zeros(3 * descs[0].n_vertices), n_steps=1)
    vo = b.offsets["vertices"]
    assert np.array_equal(xb[: 3 * vo[1]], x0)  # the first part keeps its unregularised factor
    assert s0.info()["factor_regularisation"] == 0.0
    s0.close()
    b.close()


def test_split_refactorisation_levels_match_one_launch():
    """The top levels of the tree (few supernodes) refactor split over four
    launches with several CTAs per supernode; every factor entry sees the same
    operations as in the one-CTA-per-supernode kernel: forward and adjoint
    agree bit for bit with the split switched off."""
    d = S.inverse_stiffness()
    out = []
    for split in (1, 0):
        g = Scene(d)
        g.solve_mode("persistent")
        g.set_option("split_factor", split)
        g.set_materials(np.asarray(d.youngs), np.asarray(d.poisson))
        x = d.x0.reshape(-1).copy()
        xo, vo = g.forward(x, np.zeros_like(x), n_steps=3)
        gr = g.backward(np.ones_like(x), np.zeros_like(x))
        out.append((xo, vo, gr["x"], gr["E"]))
        g.close()
    for a, b in zip(*out):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("builder", ["inverse_stiffness", "muscle_beam"])
def test_thread_and_warp_gathers_agree_bit_for_bit(builder):
    """The per-vertex sums of the local step's slots: one warp per vertex
    (small scenes) or one thread per vertex emulating the warp's lanes and
    reduction tree (large scenes); forced either way, forward and adjoint
    agree bit for bit."""
    d = {"inverse_stiffness": S.inverse_stiffness, "muscle_beam": S.muscle_beam}[builder]()
    act = np.random.default_rng(3).uniform(0, 1, (3, d.n_segments)) if d.n_segments else None
    out = []
    for form in (1, 2):
        g = Scene(d)
        g.set_option("gather", form)
        x = d.x0.reshape(-1).copy()
        xo, vo = g.forward(x, 0.01 * np.ones_like(x), n_steps=3, act=act)
        gr = g.backward(np.ones_like(x), np.zeros_like(x))
        out.append([xo, vo] + [gr[k] for k in ("x", "v", "E", "nu", "act")])
        g.close()
    for a, b in zip(*out):
        assert np.array_equal(a, b)
