"""The forms of the global solve (one launch per elimination-tree level, one
persistent launch whose CTAs claim supernodes in dependency order, level
kernels below a cut level and the persistent launch above it, one
thread-block cluster walking the levels, or one cluster holding the whole
factor in its distributed shared memory) run the same arithmetic per
supernode, so a step, its gradient and a batch agree bit for bit whichever
form the autotuner picked."""
import dataclasses

import numpy as np
import pytest

from diff_fem_b200 import scene as S
from diff_fem_b200.engine import Scene

pytestmark = pytest.mark.gpu


def run(sc, d, n, mode, act=None):
    assert sc.solve_mode(mode)["mode"] == mode
    x = np.concatenate([q.x0.reshape(-1) for q in d]) if isinstance(d, list) else d.x0.reshape(-1)
    xo, vo = sc.forward(x, np.zeros_like(x), n_steps=n, act=act)
    rng = np.random.default_rng(5)
    g = sc.backward(rng.standard_normal(x.size), rng.standard_normal(x.size))
    return xo, vo, g, sc.iterations(n)


@pytest.mark.parametrize("builder", ["inverse_stiffness", "muscle_beam", "cloth_sheet"])
def test_persistent_solve_matches_level_kernels(builder):
    d = {"inverse_stiffness": lambda: S.inverse_stiffness(nx=20, ny=6, nz=6),
         "muscle_beam": S.muscle_beam, "cloth_sheet": lambda: S.cloth_sheet(nv=12)}[builder]()
    sc = Scene(d)
    info = sc.solve_mode()
    assert info["mode"] in ("levels", "persistent", "split", "cluster", "resident", "dense")
    assert info["ms_levels"] > 0 and info["ms_persistent"] > 0
    assert info["split_level"] > 0 and info["ms_split"] > 0  # these factors have more than one level
    assert info["ms_cluster"] > 0  # few supernodes: the cluster form is a candidate
    assert info["ms_resident"] > 0  # small factors: the resident form is a candidate
    act = np.random.default_rng(1).uniform(0, 1, (4, d.n_segments)) if d.n_segments else None
    a = run(sc, d, 4, "levels", act)
    for form in ("persistent", "split", "cluster", "resident"):
        b = run(sc, d, 4, form, act)
        for u, w in zip(a[:2], b[:2]):
            assert np.array_equal(u, w), form
        for k in a[2]:
            assert np.array_equal(a[2][k], b[2][k]), (form, k)
        assert np.array_equal(a[3], b[3]), form
    sc.close()


def test_persistent_solve_in_a_batch_with_converged_parts():
    descs = [dataclasses.replace(q, time_step=1.0 / 60.0, max_iterations=15)
             for q in (S.inverse_stiffness(nx=10, ny=3, nz=3), S.cantilever(), S.muscle_beam())]
    sc = Scene.batch(descs)
    act = np.random.default_rng(2).uniform(0, 1, (3, sc.nseg))
    a = run(sc, descs, 3, "levels", act)
    for form in ("persistent", "split", "cluster"):
        b = run(sc, descs, 3, form, act)
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]), form
        for k in a[2]:
            assert np.array_equal(a[2][k], b[2][k]), (form, k)
        assert np.array_equal(a[3], b[3]), form
    sc.close()


def test_batch_tail_selection_matches_fixed_form():
    """After an autotune a batch may switch each iteration's solve to the
    persistent form once few parts are left; the result is that of a fixed form."""
    from diff_fem_b200 import _capi
    descs, _ = S.uneven_batch(n_scenes=24, t_hi=8e3, precision=_capi.DFEM_PREC_FP64, ground=False)
    sc = Scene.batch(descs)
    act = np.random.default_rng(3).uniform(0, 1, (3, sc.nseg))
    info = sc.solve_mode("auto")
    assert info["ms_largest_part_only"][1] > 0 or info["mode"] == "persistent"
    x = np.concatenate([q.x0.reshape(-1) for q in descs])
    xa, va = sc.forward(x, np.zeros_like(x), n_steps=3, act=act)
    rng = np.random.default_rng(5)
    gx, gv = rng.standard_normal(x.size), rng.standard_normal(x.size)
    ga = sc.backward(gx, gv)
    b = run(sc, descs, 3, "levels", act)
    assert np.array_equal(xa, b[0]) and np.array_equal(va, b[1])
    rng = np.random.default_rng(5)
    gb = sc.backward(rng.standard_normal(x.size), rng.standard_normal(x.size))
    for k in ga:
        assert np.array_equal(ga[k], gb[k]), k
    sc.close()


def test_resident_solve_on_the_inverse_stiffness_beam():
    """The 12,800-tet beam (213 supernodes, 10 levels): its factor fits the
    shared memory of one 16-CTA cluster; 6 steps forward and adjoint agree bit
    for bit with the persistent form."""
    d = S.inverse_stiffness()
    sc = Scene(d)
    info = sc.solve_mode()
    assert info["ms_resident"] > 0
    a = run(sc, d, 6, "persistent")
    b = run(sc, d, 6, "resident")
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    for k in a[2]:
        assert np.array_equal(a[2][k], b[2][k]), k
    assert np.array_equal(a[3], b[3])
    sc.close()


@pytest.mark.parametrize("builder", ["inverse_stiffness", "muscle_beam", "cloth_sheet"])
def test_dense_inverse_form_matches_the_triangular_solves(builder):
    """The dense-inverse form (X = Hs^-1 from the factor, one product per
    solve) agrees with the supernodal triangular solves to rounding, forward
    and adjoint, is deterministic, and follows a material update."""
    d = {"inverse_stiffness": lambda: S.inverse_stiffness(nx=20, ny=6, nz=6),
         "muscle_beam": S.muscle_beam, "cloth_sheet": lambda: S.cloth_sheet(nv=12)}[builder]()
    sc = Scene(d)
    assert sc.solve_mode()["ms_dense"] > 0  # single small scenes: a candidate
    act = np.random.default_rng(1).uniform(0, 1, (4, d.n_segments)) if d.n_segments else None
    a = run(sc, d, 4, "persistent", act)
    b = run(sc, d, 4, "dense", act)
    c = run(sc, d, 4, "dense", act)

    def rel(u, w):
        return np.abs(u - w).max() / max(np.abs(w).max(), 1e-300)

    assert rel(b[0], a[0]) < 1e-12 and rel(b[1], a[1]) < 1e-10
    for k in a[2]:
        if a[2][k].size:
            assert rel(b[2][k], a[2][k]) < 1e-9, k
    assert np.array_equal(a[3], b[3])
    for u, w in zip(b[:2], c[:2]):
        assert np.array_equal(u, w)
    for k in b[2]:
        assert np.array_equal(b[2][k], c[2][k]), k
    if d.n_tets:
        E = np.asarray(d.youngs) * np.random.default_rng(2).uniform(0.5, 2.0, d.n_tets)
        sc.set_materials(E, d.poisson)
        e = run(sc, d, 4, "dense", act)
        f = run(sc, d, 4, "persistent", act)
        assert rel(e[0], f[0]) < 1e-12 and not np.array_equal(e[0], b[0])
    sc.close()


def test_dense_inverse_form_is_refused_for_batches():
    from diff_fem_b200 import _capi
    descs = [dataclasses.replace(q, time_step=1.0 / 60.0, max_iterations=15) for q in (S.cantilever(), S.muscle_beam())]
    sc = Scene.batch(descs)
    assert sc.solve_mode()["ms_dense"] == 0
    with pytest.raises(_capi.DfemError) as ex:
        sc.solve_mode("dense")
    assert ex.value.code == _capi.DFEM_ERR_INVALID
    sc.close()
