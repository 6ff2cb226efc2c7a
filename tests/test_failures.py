"""Failure detection on the GPU without a GPU fault: every capped loop or
bounded wait of the engine, lowered through dfem_set_limit until the scene
meets it, makes the call return DFEM_ERR_CAP through the device status word;
the kernels finish normally and the same handle then reproduces a clean run.
Allocation failures are injected on the host (dfem_debug_fail_allocations)
and come back as DFEM_ERR_NOMEM, again leaving the handle or the next
creation usable."""
import numpy as np
import pytest

from diff_fem_b200 import _capi, scene as S
from diff_fem_b200.engine import Scene

pytestmark = pytest.mark.gpu


def expect_cap(fn):
    with pytest.raises(_capi.DfemError) as ex:
        fn()
    assert ex.value.code == _capi.DFEM_ERR_CAP, str(ex.value)
    return str(ex.value)


def run(sc, d, n, v=None):
    x = d.x0.reshape(-1).copy()
    v = np.zeros_like(x) if v is None else v
    xo, vo = sc.forward(x, v, n_steps=n)
    g = sc.backward(np.ones_like(x), np.zeros_like(x))
    return xo, vo, g["x"]


@pytest.mark.parametrize("which,scene", [("contact_passes", "box"), ("impacts_per_vertex", "box"),
                                         ("soft_impacts_per_vertex", "cloth"), ("group_members", "cloth")])
def test_contact_caps_report_and_leave_the_handle_usable(which, scene):
    if scene == "box":
        d, n = S.drop_box(), 6
        v = d.initial_velocity.copy()
    else:
        d, n = S.cloth_on_block(), 8
        v = d.initial_velocity.copy()
    sc = Scene(d)
    ref = run(sc, d, n, v)
    assert sc.contact_passes(n).sum() > 0
    sc.set_limit(which, 0)
    msg = expect_cap(lambda: run(sc, d, n, v))
    assert {"contact_passes": "pass cap", "impacts_per_vertex": "obstacle faces",
            "soft_impacts_per_vertex": "soft faces", "group_members": "members"}[which] in msg
    sc.set_limit(which)  # the built-in cap again
    again = run(sc, d, n, v)
    for a, b in zip(ref, again):
        assert np.array_equal(a, b)
    sc.close()


def test_persistent_solve_wait_bound_reports_and_leaves_the_handle_usable():
    """The persistent solve's dependency waits give up after one poll: CTAs
    raise the abort word, every CTA stops claiming work, the launch ends."""
    d = S.inverse_stiffness()
    sc = Scene(d)
    assert sc.solve_mode("persistent")["mode"] == "persistent"
    ref = run(sc, d, 3)
    sc.set_limit("solve_wait_polls", 1)
    msg = expect_cap(lambda: run(sc, d, 3))
    assert "persistent" in msg
    sc.set_limit("solve_wait_polls")
    again = run(sc, d, 3)
    for a, b in zip(ref, again):
        assert np.array_equal(a, b)
    sc.close()


def test_limits_above_the_built_in_caps_are_rejected():
    sc = Scene(S.drop_box())
    for which, cap in [("contact_passes", 64), ("impacts_per_vertex", 8), ("soft_impacts_per_vertex", 16),
                       ("group_members", 32)]:
        with pytest.raises(_capi.DfemError) as ex:
            sc.set_limit(which, cap + 1)
        assert ex.value.code == _capi.DFEM_ERR_INVALID
    sc.close()


def test_injected_allocation_failures_map_to_nomem():
    lib = _capi.lib()
    d = S.cantilever()
    failed = 0
    try:
        for after in (0, 2, 7, 20, 60):
            lib.dfem_debug_fail_allocations(after)
            try:
                Scene(d).close()
            except _capi.DfemError as ex:
                assert ex.code == _capi.DFEM_ERR_NOMEM, str(ex)
                failed += 1
    finally:
        lib.dfem_debug_fail_allocations(-1)
    assert failed >= 3
    sc = Scene(d)  # creation works again
    ref = run(sc, d, 4)
    # a forward that needs more per-step buffers fails to allocate them; the handle stays usable
    lib.dfem_debug_fail_allocations(1)
    try:
        with pytest.raises(_capi.DfemError) as ex:
            run(sc, d, 40)
        assert ex.value.code == _capi.DFEM_ERR_NOMEM
    finally:
        lib.dfem_debug_fail_allocations(-1)
    again = run(sc, d, 4)
    for a, b in zip(ref, again):
        assert np.array_equal(a, b)
    sc.close()


def test_record_store_allocation_failure_falls_back_to_replays():
    """A forward whose contact-record store cannot grow runs without
    recording, and the adjoint replays its contact steps: the gradients equal
    those of a run that replays every step, bit for bit, wherever among the
    store's arrays the allocation fails."""
    lib = _capi.lib()
    d = S.drop_box(mu=0.3)
    n = 4
    x = d.x0.reshape(-1).copy()
    v = np.tile([1.0, -1.0, 0.3], d.n_vertices)
    rng = np.random.default_rng(8)
    gx, gv = rng.standard_normal(x.size), rng.standard_normal(x.size)
    ref = Scene(d)
    ref.set_adjoint_budget(0)
    ref.forward(x, v, n_steps=n)
    assert ref.contact_passes(n).sum() > 0
    want = ref.backward(gx, gv)
    ref.close()
    g = Scene(d)
    g.forward(x, v, n_steps=n)  # records every contact step; the next forward asks for a larger store
    g.backward(gx, gv)
    try:
        for after in range(5):
            lib.dfem_debug_fail_allocations(after)
            g.forward(x, v, n_steps=n)
            lib.dfem_debug_fail_allocations(-1)
            got = g.backward(gx, gv)
            for k in ("x", "v", "E", "nu"):
                assert np.array_equal(got[k], want[k]), (after, k)
    finally:
        lib.dfem_debug_fail_allocations(-1)
    g.forward(x, v, n_steps=n)
    got = g.backward(gx, gv)
    for k in ("x", "v", "E", "nu"):
        assert np.array_equal(got[k], want[k]), k
    g.close()
