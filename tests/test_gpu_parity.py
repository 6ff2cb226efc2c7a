"""GPU parity: the CUDA engine (through the C ABI) against the CPU FP64 oracle.

Tolerances (plain FP64 form): positions and velocities within 1e-9 relative
to the oracle's scale, gradients within 1e-8 relative, iteration counts equal.
"""
import dataclasses

import numpy as np
import pytest

from diff_fem_b200 import _capi, scene as S
from diff_fem_b200.engine import Scene
from oracle import oracle as O

pytestmark = pytest.mark.gpu

POS_TOL = 1e-9
GRAD_TOL = 1e-8


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def run_both(d, n_steps, act=None, x=None, v=None, seed=0):
    rng = np.random.default_rng(seed)
    if x is None:
        x = d.x0.reshape(-1).copy()
    if v is None:
        v = np.zeros_like(x)
    g = Scene(d)
    o = O.OracleScene(d)
    xg, vg, tg = g.forward(x, v, n_steps=n_steps, act=act, traj=True)
    ro = o.forward(x, v, n_steps=n_steps, act=act, traj=True)
    return g, o, (xg, vg, tg), ro


def test_cantilever_forward_100_steps():
    d = S.cantilever()
    g, o, (xg, vg, tg), ro = run_both(d, 100)
    assert np.array_equal(g.iterations(100), ro["iters"])
    assert rel(tg, ro["traj"]) < POS_TOL
    assert rel(xg, ro["x"]) < POS_TOL
    assert rel(vg, ro["v"]) < POS_TOL


def test_inverse_stiffness_forward_and_adjoint():
    d = S.inverse_stiffness()
    n = 4
    g, o, (xg, vg, tg), ro = run_both(d, n)
    assert np.array_equal(g.iterations(n), ro["iters"])
    assert rel(tg, ro["traj"]) < POS_TOL
    rng = np.random.default_rng(1)
    gx, gv = rng.standard_normal(xg.size), rng.standard_normal(xg.size)
    bg = g.backward(gx, gv)
    bo = o.backward(gx, gv)
    for k in ("x", "v", "E", "nu"):
        assert rel(bg[k], bo[k]) < GRAD_TOL, k


def test_muscles_forward_and_adjoint():
    d = S.muscle_beam()
    n = 5
    act = np.random.default_rng(2).uniform(0, 1, (n, d.n_segments))
    g, o, (xg, vg, tg), ro = run_both(d, n, act=act)
    assert np.array_equal(g.iterations(n), ro["iters"])
    assert rel(tg, ro["traj"]) < POS_TOL
    rng = np.random.default_rng(3)
    gx, gv = rng.standard_normal(xg.size), rng.standard_normal(xg.size)
    bg, bo = g.backward(gx, gv), o.backward(gx, gv)
    for k in ("x", "v", "E", "nu", "act"):
        assert rel(bg[k], bo[k]) < GRAD_TOL, k


def test_pneumatic_springs_forward_and_adjoint():
    """Pneumatic springs (PneumaticConstraint: length rest * activation) on
    their own activation channels after one muscle chain's segments: positions,
    and gradients including dL/d(activation) of both kinds of channel; then
    the default activations (muscles 0, pneumatic channels 1)."""
    d = S.pneumatic_beam()
    n = 5
    act = np.random.default_rng(12).uniform(0.6, 1.4, (n, d.n_segments))
    g, o, (xg, vg, tg), ro = run_both(d, n, act=act)
    assert np.array_equal(g.iterations(n), ro["iters"])
    assert rel(tg, ro["traj"]) < POS_TOL
    rng = np.random.default_rng(13)
    gx, gv = rng.standard_normal(xg.size), rng.standard_normal(xg.size)
    bg, bo = g.backward(gx, gv), o.backward(gx, gv)
    for k in ("x", "v", "E", "nu", "act"):
        assert rel(bg[k], bo[k]) < GRAD_TOL, k
    assert np.abs(bg["act"][:, 2:]).max() > 0  # the pneumatic channels
    x = d.x0.reshape(-1).copy()
    xg, vg = g.forward(x, np.zeros_like(x), n_steps=3)
    ro = o.forward(x, np.zeros_like(x), n_steps=3)
    assert rel(xg, ro["x"]) < POS_TOL
    g.close()


def test_cloth_forward_and_adjoint():
    d = S.cloth_sheet(nv=10)
    n = 6
    g, o, (xg, vg, tg), ro = run_both(d, n)
    assert np.array_equal(g.iterations(n), ro["iters"])
    assert rel(tg, ro["traj"]) < POS_TOL
    rng = np.random.default_rng(4)
    gx, gv = rng.standard_normal(xg.size), rng.standard_normal(xg.size)
    bg, bo = g.backward(gx, gv), o.backward(gx, gv)
    for k in ("x", "v"):
        assert rel(bg[k], bo[k]) < GRAD_TOL, k


def test_device_pointers_match_host_path_and_are_deterministic():
    import torch
    d = S.inverse_stiffness(nx=12, ny=4, nz=4)
    g = Scene(d)
    x = d.x0.reshape(-1).copy()
    v = np.zeros_like(x)
    xh, vh = g.forward(x, v, n_steps=3)
    xd, vd = g.forward(torch.tensor(x, device="cuda"), torch.tensor(v, device="cuda"), n_steps=3)
    assert np.array_equal(xh, xd.cpu().numpy()) and np.array_equal(vh, vd.cpu().numpy())
    xh2, vh2 = g.forward(x, v, n_steps=3)
    assert np.array_equal(xh, xh2) and np.array_equal(vh, vh2)


def test_set_materials_refactors():
    d = S.inverse_stiffness(nx=10, ny=3, nz=3)
    g = Scene(d)
    o = O.OracleScene(d)
    E2 = S.log_uniform_moduli(d.n_tets, 5678)
    g.set_materials(E2, d.poisson)
    o.set_materials(E2, d.poisson)
    x = d.x0.reshape(-1).copy()
    xg, vg = g.forward(x, np.zeros_like(x), n_steps=5)
    ro = o.forward(x, np.zeros_like(x), n_steps=5)
    assert rel(xg, ro["x"]) < POS_TOL


@pytest.mark.parametrize("mu", [1.0, 0.3])
def test_obstacle_contact_forward(mu):
    """Soft box dropped on a ground quad: CCD, Coulomb-cone reaction, Jacobi contact iterations."""
    d = S.drop_box(mu=mu)
    n = 30
    x = d.x0.reshape(-1).copy()
    v = d.initial_velocity.copy()
    g = Scene(d)
    o = O.OracleScene(d)
    xg, vg, tg = g.forward(x, v, n_steps=n, traj=True)
    ro = o.forward(x, v, n_steps=n, traj=True)
    assert np.array_equal(g.contact_passes(n), o.contact_passes())
    assert o.contact_passes().sum() > 0
    assert np.array_equal(g.iterations(n), ro["iters"])
    assert rel(tg, ro["traj"]) < POS_TOL


@pytest.mark.parametrize("case", ["small", "wide", "no_ground"])
def test_soft_contact_forward(case):
    """Soft-soft contact (self-collision on): a cloth dropped onto a soft block
    that rests on a ground quad.  Soft CCD both ways (cloth vertices on block
    faces, block vertices on cloth faces), face groups with the stick/slide
    exchange, the self forces remembered between the iterations of a step,
    and the block's obstacle contacts, against the oracle."""
    if case == "small":
        d, n = S.cloth_on_block(), 10
    elif case == "wide":
        d, n = S.cloth_on_block(nv=8, edge=0.0071, block=(3, 1, 3), block_edge=0.02), 8
    else:  # soft contact only: no obstacle face at all (the block falls too)
        d, n = S.cloth_on_block(), 8
        v0 = d.initial_velocity
        d = dataclasses.replace(d, obstacle_x=np.zeros((0, 3)), obstacle_faces=np.zeros((0, 3), np.int32))
        d.initial_velocity = v0
    x = d.x0.reshape(-1).copy()
    v = d.initial_velocity.copy()
    g = Scene(d)
    o = O.OracleScene(d)
    xg, vg, tg = g.forward(x, v, n_steps=n, traj=True)
    ro = o.forward(x, v, n_steps=n, traj=True)
    assert o.contact_passes().sum() > 0
    assert np.array_equal(g.contact_passes(n), o.contact_passes())
    assert np.array_equal(g.iterations(n), ro["iters"])
    assert rel(tg, ro["traj"]) < POS_TOL
    assert rel(vg, ro["v"]) < POS_TOL
    g.close()


def test_soft_contact_steps_carry_no_remembered_forces():
    """Every step starts with zero remembered contact forces
    (World::TimeStepping -> updateCollisionScene, World.h:700,742-753): a
    3-step forward equals three 1-step forwards bit for bit, on the GPU as in
    the oracle."""
    d = S.cloth_on_block()
    x = d.x0.reshape(-1).copy()
    v = d.initial_velocity.copy()
    g = Scene(d)
    x3, v3 = g.forward(x, v, n_steps=3)
    xs, vs = x, v
    passes = 0
    for _ in range(3):
        xs, vs = g.forward(xs, vs, n_steps=1)
        passes += int(g.contact_passes(1).sum())
    assert passes > 0
    assert np.array_equal(x3, xs) and np.array_equal(v3, vs)
    g.close()


def test_scene_created_after_a_larger_one_leaves_its_kernels_usable():
    """The kernels' shared-memory limits are process-wide: a small scene
    created after a large one must not lower them under the large scene's
    launches (refactorisation, solves, autotune)."""
    big = S.inverse_stiffness()
    g_big = Scene(big)
    x = big.x0.reshape(-1).copy()
    v = np.zeros_like(x)
    x_ref, v_ref = g_big.forward(x, v, n_steps=2)
    small = S.inverse_stiffness(nx=4, ny=2, nz=2)
    g_small = Scene(small)
    xs = small.x0.reshape(-1).copy()
    g_small.forward(xs, np.zeros_like(xs), n_steps=2)
    g_big.set_materials(big.youngs, big.poisson)
    x2, v2 = g_big.forward(x, v, n_steps=2)
    assert np.array_equal(x2, x_ref) and np.array_equal(v2, v_ref)
    g_big.solve_mode("auto")
    x3, _ = g_big.forward(x, v, n_steps=2)
    assert np.array_equal(x3, x_ref)
    g_small.close()
    g_big.close()


@pytest.mark.parametrize("case,every", [("small", 1), ("small", 2), ("wide", 1), ("ball", 1)])
def test_soft_contact_adjoint(case, every):
    """Adjoint of soft-soft contact (group exchange reversed per computed
    iteration, the remembered self forces' cotangent carried between the
    iterations of a step, checkpoints every step or every second step)
    against the oracle's
    adjoint (forward-mode duals per group; pinned by central differences)."""
    if case == "small":
        d, n = S.cloth_on_block(), 4
    elif case == "wide":
        d, n = S.cloth_on_block(nv=8, edge=0.0071, block=(3, 1, 3), block_edge=0.02), 3
    else:  # a cloth draping over a small soft ball on the ground
        d, n = S.cloth_on_soft_ball(nv=12, edge=0.02, radius=0.08, drop=0.03, subdiv=2), 14
        d.initial_velocity = np.zeros(3 * d.n_vertices)
    v = d.initial_velocity.copy()
    d = dataclasses.replace(d, checkpoint_every=every)
    x = d.x0.reshape(-1).copy()
    g = Scene(d)
    o = O.OracleScene(d)
    xg, vg = g.forward(x, v, n_steps=n)
    ro = o.forward(x, v, n_steps=n)
    assert o.contact_passes().sum() > 0
    assert np.array_equal(g.contact_passes(n), o.contact_passes())
    assert rel(xg, ro["x"]) < POS_TOL
    rng = np.random.default_rng(6)
    gx, gv = rng.standard_normal(x.size), rng.standard_normal(x.size)
    bg, bo = g.backward(gx, gv), o.backward(gx, gv)
    for k in ("x", "v", "E"):
        assert rel(bg[k], bo[k]) < GRAD_TOL, (k, rel(bg[k], bo[k]))
    g.close()


@pytest.mark.parametrize("case", ["drop", "slide"])
def test_obstacle_contact_adjoint(case):
    """Adjoint through the contact phase (Jacobi sweeps, friction cone,
    relaxation) against the oracle's restatement: x, v, E, nu gradients.
    "slide" lands with a tangential velocity, so the friction cone clamps."""
    d = S.drop_box(mu=0.3)
    n = 6
    x = d.x0.reshape(-1).copy()
    v = d.initial_velocity.copy() if case == "drop" else np.tile([1.0, -1.0, 0.3], d.n_vertices)
    g = Scene(d)
    o = O.OracleScene(d)
    xg, vg = g.forward(x, v, n_steps=n)
    o.forward(x, v, n_steps=n)
    assert g.contact_passes(n).sum() > 0
    rng = np.random.default_rng(7)
    gx, gv = rng.standard_normal(x.size), rng.standard_normal(x.size)
    bg, bo = g.backward(gx, gv), o.backward(gx, gv)
    for k in ("x", "v", "E", "nu"):
        assert rel(bg[k], bo[k]) < GRAD_TOL, (k, rel(bg[k], bo[k]))
    # a second backward of the same forward gives the same result
    bg2 = g.backward(gx, gv)
    assert np.array_equal(bg["x"], bg2["x"]) and np.array_equal(bg["E"], bg2["E"])


@pytest.mark.parametrize("builder", ["cantilever", "muscle_beam", "cloth_sheet"])
def test_eval_local_matches_oracle(builder):
    d = getattr(S, builder)()
    g = Scene(d)
    o = O.OracleScene(d)
    rng = np.random.default_rng(9)
    x = d.x0.reshape(-1) + 0.01 * rng.standard_normal(3 * d.n_vertices)
    act = rng.uniform(0, 1, d.n_segments) if d.n_segments else None
    if act is not None:
        g.set_activations(act)
    assert rel(g.eval_local(x), o.eval_local(x, act)) < POS_TOL


def test_backward_before_forward_is_a_state_error():
    d = S.cantilever()
    g = Scene(d)
    with pytest.raises(_capi.DfemError) as e:
        g.backward(np.zeros(3 * d.n_vertices), np.zeros(3 * d.n_vertices))
    assert e.value.code == 5


def test_nonfinite_input_reports_status():
    d = S.cantilever()
    g = Scene(d)
    x = d.x0.reshape(-1).copy()
    x[7] = np.nan
    with pytest.raises(_capi.DfemError) as e:
        g.forward(x, np.zeros_like(x), n_steps=1)
    assert e.value.code == 4
    # the context stays usable
    xg, _ = g.forward(d.x0.reshape(-1).copy(), np.zeros_like(x), n_steps=1)
    assert np.all(np.isfinite(xg))


def test_muscle_star_on_ground_forward_and_adjoint():
    """The muscle star resting on its ground quad: activations drive the arms,
    the contact phase runs every step, and the activation gradient flows
    through it."""
    d = S.muscle_star(refine=1, ground=True, mu=0.5)
    n = 4
    act = np.repeat(np.random.default_rng(42).uniform(0, 1, (n, d.n_segments // 6)), 6, axis=1)
    g, o, (xg, vg, tg), ro = run_both(d, n, act=act)
    assert g.contact_passes(n).sum() > 0
    assert np.array_equal(g.contact_passes(n), o.contact_passes())
    assert np.array_equal(g.iterations(n), ro["iters"])
    assert rel(tg, ro["traj"]) < POS_TOL
    rng = np.random.default_rng(9)
    gx, gv = rng.standard_normal(xg.size), rng.standard_normal(xg.size)
    bg, bo = g.backward(gx, gv), o.backward(gx, gv)
    for k in ("x", "v", "E", "act"):
        assert rel(bg[k], bo[k]) < GRAD_TOL, (k, rel(bg[k], bo[k]))


def test_stored_and_recomputed_iterates_give_identical_gradients():
    """The adjoint reads the stored iterates of every step, or replays each
    step from its checkpoint when the memory budget is too small: the same
    arithmetic, bit for bit."""
    d = S.muscle_beam()
    n = 5
    act = np.random.default_rng(4).uniform(0, 1, (n, d.n_segments))
    x = d.x0.reshape(-1).copy()
    rng = np.random.default_rng(6)
    gx, gv = rng.standard_normal(x.size), rng.standard_normal(x.size)
    out = []
    for budget in (1 << 31, 0):
        g = Scene(d)
        g.set_adjoint_budget(budget)
        g.forward(x, np.zeros_like(x), n_steps=n, act=act)
        out.append(g.backward(gx, gv))
        g.close()
    for k in ("x", "v", "E", "nu", "act"):
        assert np.array_equal(out[0][k], out[1][k]), k


def test_cloth_on_ball_forward_and_adjoint():
    """Cloth (springs, bending, gravity) dropped on a ball (static obstacle
    surface) above a ground quad: the contact phase with many contact
    vertices, and its adjoint with respect to the initial velocities."""
    d = S.cloth_on_ball(nv=10, radius=0.05, drop=0.004, subdiv=2)
    n = 12
    g, o, (xg, vg, tg), ro = run_both(d, n)
    assert g.contact_passes(n).sum() > 0
    assert np.array_equal(g.contact_passes(n), o.contact_passes())
    assert np.array_equal(g.iterations(n), ro["iters"])
    assert rel(tg, ro["traj"]) < POS_TOL
    rng = np.random.default_rng(10)
    gx, gv = rng.standard_normal(xg.size), rng.standard_normal(xg.size)
    bg, bo = g.backward(gx, gv), o.backward(gx, gv)
    for k in ("x", "v"):
        assert rel(bg[k], bo[k]) < GRAD_TOL, (k, rel(bg[k], bo[k]))


@pytest.mark.parametrize("form", ["levels", "persistent"])
def test_streamed_blocks_forward_and_adjoint(form):
    """A 16x16x16-cube block (20,480 tets): its top supernodes' below-diagonal
    blocks exceed the shared memory and are streamed through it in column
    chunks, in both solve forms; against the oracle at the FP64 tolerances."""
    d = S.inverse_stiffness(nx=16, ny=16, nz=16)
    g = Scene(d)
    assert g.solve_mode(form)["mode"] == form
    o = O.OracleScene(d)
    x = d.x0.reshape(-1).copy()
    v = 0.05 * np.random.default_rng(1).standard_normal(x.size)
    n = 3
    xg, vg = g.forward(x, v, n_steps=n)
    ro = o.forward(x, v, n_steps=n)
    assert np.array_equal(g.iterations(n), ro["iters"])
    assert rel(xg, ro["x"]) < POS_TOL and rel(vg, ro["v"]) < POS_TOL
    rng = np.random.default_rng(2)
    gx, gv = rng.standard_normal(xg.size), rng.standard_normal(xg.size)
    bg, bo = g.backward(gx, gv), o.backward(gx, gv)
    for k in ("x", "v", "E"):
        assert rel(bg[k], bo[k]) < GRAD_TOL, k
    g.close()


def test_underwater_drag_forward_and_adjoint():
    """Underwater drag and lift on the surface faces (per-face forces from the
    step's start state, gathered per vertex into v_wc) and their adjoint,
    against the oracle at the FP64 tolerances."""
    d, v0 = S.underwater_block()
    g = Scene(d)
    o = O.OracleScene(d)
    x = d.x0.reshape(-1).copy()
    v = v0.reshape(-1).copy()
    n = 4
    xg, vg = g.forward(x, v, n_steps=n)
    ro = o.forward(x, v, n_steps=n)
    assert np.array_equal(g.iterations(n), ro["iters"])
    assert rel(xg, ro["x"]) < POS_TOL and rel(vg, ro["v"]) < POS_TOL
    rng = np.random.default_rng(4)
    gx, gv = rng.standard_normal(xg.size), rng.standard_normal(xg.size)
    bg, bo = g.backward(gx, gv), o.backward(gx, gv)
    for k in ("x", "v", "E"):
        assert rel(bg[k], bo[k]) < GRAD_TOL, k
    g.close()


def test_contact_records_from_the_forward_match_replays():
    """With every step's iterates stored, the forward also records the contact
    iterations of its contact steps (as many as the adjoint budget holds; the
    rest are replayed by the adjoint, after the forward's records).  The
    first call (room for few records: most contact steps replayed), a second
    call (room grown to all of them: none replayed) and a run that replays
    every step give the same gradients, bit for bit."""
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
    for _ in range(2):
        g.forward(x, v, n_steps=n)
        got = g.backward(gx, gv)
        for k in ("x", "v", "E", "nu"):
            assert np.array_equal(got[k], want[k]), k
    g.close()


@pytest.mark.parametrize("case", ["muscle_beam", "drop_box", "underwater"])
@pytest.mark.parametrize("budget", [None, 0])
def test_checkpoints_every_k_steps_give_identical_gradients(case, budget):
    """checkpoint_every = 3: the forward keeps the start state of every third
    step only, and the adjoint regenerates each segment's states from its
    checkpoint before reversing it (with the iterates stored or replayed, with
    contact and with drag).  The same arithmetic as checkpoints at every
    step: identical results, bit for bit (7 steps: a partial last segment)."""
    import dataclasses
    n = 7
    if case == "muscle_beam":
        d = S.muscle_beam()
        v = np.zeros(3 * d.n_vertices)
    elif case == "drop_box":
        d = S.drop_box(mu=0.3)
        v = np.tile([1.0, -1.0, 0.3], d.n_vertices)
    else:
        d, v0 = S.underwater_block()
        v = v0.reshape(-1).copy()
    act = np.random.default_rng(4).uniform(0, 1, (n, d.n_segments)) if d.n_segments else None
    x = d.x0.reshape(-1).copy()
    rng = np.random.default_rng(12)
    gx, gv = rng.standard_normal(x.size), rng.standard_normal(x.size)
    out = []
    for k in (1, 3):
        g = Scene(dataclasses.replace(d, checkpoint_every=k))
        if budget is not None:
            g.set_adjoint_budget(budget)
        xo, vo = g.forward(x, v, n_steps=n, act=act)
        out.append((xo, vo, g.backward(gx, gv)))
        g.close()
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])
    for key in out[0][2]:
        assert np.array_equal(out[0][2][key], out[1][2][key]), key


@pytest.mark.parametrize("name,pre", [("bridgesus", 0), ("baymax", 20), ("cloth_ball", 68), ("octopus", 0),
                                      ("droneman", 0)])
def test_reference_data_scenes_forward_and_adjoint(name, pre):
    """Five of diff_fem's own data scenes (tests/golden/ref_scenes, written by
    make_ref_scenes.py from its data directory): 10 steps forward and adjoint
    against the oracle (droneman: its 48 pneumatic springs on random
    activations).  baymax and cloth_ball start from the oracle's state
    `pre` steps in, a few steps before their first contact, so the window
    holds contact passes (baymax: the ground obstacle; cloth_ball: soft-soft
    contact with the ball)."""
    import os
    d = S.load_npz(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_scenes", name + ".npz"))
    x = d.x0.reshape(-1).copy()
    v = np.tile([0.3, 0.0, 0.0], d.n_vertices) if d.underwater else np.zeros_like(x)
    o = O.OracleScene(d)
    if pre:
        r = o.forward(x, v, n_steps=pre)
        x, v = r["x"], r["v"]
    rng = np.random.default_rng(21)
    act = rng.uniform(0, 1, (10, d.n_segments)) if d.n_segments else None
    g = Scene(d)
    xg, vg, tg = g.forward(x, v, n_steps=10, act=act, traj=True)
    ro = o.forward(x, v, n_steps=10, act=act, traj=True)
    if name in ("baymax", "cloth_ball"):
        assert o.contact_passes().sum() > 0
        assert np.array_equal(g.contact_passes(10), o.contact_passes())
    assert np.array_equal(g.iterations(10), ro["iters"])
    assert rel(tg, ro["traj"]) < POS_TOL
    assert rel(vg, ro["v"]) < POS_TOL
    gx, gv = rng.standard_normal(x.size), rng.standard_normal(x.size)
    bg, bo = g.backward(gx, gv), o.backward(gx, gv)
    for k in ("x", "v", "E") + (("act",) if d.n_segments else ()):
        assert rel(bg[k], bo[k]) < GRAD_TOL, (k, rel(bg[k], bo[k]))
    g.close()


def test_obstacle_broad_phase_matches_testing_every_face():
    """The obstacle detection's broad phase (a uniform grid over the static
    obstacle faces) drops no impact: trajectories, contact passes and
    gradients are bit-identical to testing every face (broad-phase cell
    limit 0), on a cloth falling on a 1,280-face ball."""
    d = S.cloth_on_ball(nv=16, radius=0.08, drop=0.01, subdiv=3)
    x = d.x0.reshape(-1).copy()
    v = np.zeros_like(x)
    n = 16
    rng = np.random.default_rng(8)
    gx, gv = rng.standard_normal(x.size), rng.standard_normal(x.size)
    out = []
    for cells in (-1, 0):
        g = Scene(d)
        g.set_limit("broad_phase_cells", cells)
        xg, vg, tg = g.forward(x, v, n_steps=n, traj=True)
        passes = g.contact_passes(n)
        b = g.backward(gx, gv)
        out.append((tg, vg, passes, b["x"], b["v"]))
        g.close()
    assert out[0][2].sum() > 0
    for a, b in zip(out[0], out[1]):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("case", ["box", "star", "cloth"])
def test_fused_contact_phase_matches_the_loop_of_kernels(case):
    """The obstacle contact phase as one cooperative launch (the default)
    gives the same trajectories, contact passes, iteration counts and
    gradients, bit for bit, as the conditional graph loop of kernels."""
    if case == "box":
        d, n = S.drop_box(), 6
        v = d.initial_velocity.copy()
        act = None
    elif case == "star":
        d, n = S.muscle_star(refine=1), 8
        v = None
        act = np.random.default_rng(3).uniform(0, 1, (n, d.n_segments))
    else:
        d, n = S.cloth_on_ball(nv=16, radius=0.08, drop=0.01, subdiv=3), 16
        v = None
        act = None
    x = d.x0.reshape(-1).copy()
    v = np.zeros_like(x) if v is None else v
    rng = np.random.default_rng(9)
    gx, gv = rng.standard_normal(x.size), rng.standard_normal(x.size)
    out = []
    for fused in (1, 0):
        g = Scene(d)
        g.set_option("fused_contact", fused)
        xg, vg, tg = g.forward(x, v, n_steps=n, act=act, traj=True)
        res = [tg, vg, g.contact_passes(n), g.iterations(n)]
        b = g.backward(gx, gv)
        res += [b[k] for k in ("x", "v", "E")] + ([b["act"]] if act is not None else [])
        out.append(res)
        g.close()
    assert out[0][2].sum() > 0
    for a, b in zip(out[0], out[1]):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("case", ["articulated_beam", "baymax_skeleton"])
def test_skeleton_forward_matches_oracle(case):
    """Articulated skeleton (Link tree, World::ComputeSolution's rigid branch):
    trajectory, iteration counts and joint state (World::mJointQ / mJointQd)
    against the oracle, which solves the reference's Schur form literally
    (two Qf solves, the precomputed Qb_M - Qc_L Qf^-1 Qc_L^T); the engine uses
    the equivalent multiplier form on the step's full solve.  A second call
    continues from the joint state the first left; set_joint_state restarts
    from a given state."""
    import os
    rng = np.random.default_rng(31)
    if case == "articulated_beam":
        d = S.articulated_beam()
        n = 8
        act = np.tile([0.5, 2.0], (n, 1)) * rng.uniform(0.5, 1.5, (n, 2))
    else:
        d = S.load_npz(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_scenes",
                                    "baymax_skeleton.npz"))
        n = 10
        act = rng.uniform(-20.0, 20.0, (n, d.n_segments))
    x = d.x0.reshape(-1).copy()
    v = np.zeros_like(x)
    g, o, (xg, vg, tg), ro = run_both(d, n, act=act, x=x, v=v)
    assert np.array_equal(g.iterations(n), ro["iters"])
    assert rel(tg, ro["traj"]) < POS_TOL
    assert rel(vg, ro["v"]) < POS_TOL
    jg, jdg = g.joint_state()
    jo, jdo = o.joint_state()
    assert np.abs(jg - jo).max() < 1e-9 and np.abs(jdg - jdo).max() < 1e-9
    assert np.abs(jg[12:]).max() > 1e-3  # the torques moved the joints
    # continue from the state the first call left
    xg2, vg2 = g.forward(xg, vg, n_steps=2, act=act[:2])
    ro2 = o.forward(ro["x"], ro["v"], n_steps=2, act=act[:2])
    assert rel(xg2, ro2["x"]) < POS_TOL
    # restart from a given joint state
    g.set_joint_state(jo, jdo)
    o.set_joint_state(jo, jdo)
    xg3, _ = g.forward(ro["x"], ro["v"], n_steps=2, act=act[:2])
    ro3 = o.forward(ro["x"], ro["v"], n_steps=2, act=act[:2])
    assert rel(xg3, ro3["x"]) < POS_TOL
    g.close()


def _skeleton_case(name):
    """A skeleton scene at a fixed PD iteration count (the count then cannot
    change under the finite-difference perturbations), its start state a few
    steps in (rotated root, moved joints) and per-step torque activations."""
    import os
    rng = np.random.default_rng(41)
    if name == "articulated_beam":
        d = dataclasses.replace(S.articulated_beam(), max_iterations=6)
        act0 = np.tile([0.5, 2.0], (4, 1))
        n = 3
    else:
        d = S.load_npz(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_scenes",
                                    "baymax_skeleton.npz"))
        d = dataclasses.replace(d, max_iterations=5)
        act0 = rng.uniform(-20.0, 20.0, (4, d.n_segments))
        n = 2
    o = O.OracleScene(d)
    x = d.x0.reshape(-1).copy()
    v = np.tile([0.2, 0.1, -0.1], d.n_vertices)
    r0 = o.forward(x, v, n_steps=4, act=act0)
    jq, jqd = o.joint_state()
    act = (act0[:n] if act0.shape[0] >= n else act0) * rng.uniform(0.7, 1.3, (n, d.n_segments))
    return d, o, r0["x"], r0["v"], jq, jqd, act, n


@pytest.mark.parametrize("case", ["articulated_beam", "baymax_skeleton"])
def test_skeleton_adjoint_matches_oracle_finite_differences(case):
    """The adjoint through the links (backward_act's dq, dqd, djq, djqd and the
    joint torques' dtau, CppAD in the reference): every gradient against
    central differences of the oracle's forward along random directions of x,
    v, the joint state (jq, jqd; the root's T need not be a rotation), the
    torque activations and Young's moduli, for L = gx.x' + gv.v' + gjq.jq' +
    gjqd.jqd' after n steps."""
    d, o, x, v, jq, jqd, act, n = _skeleton_case(case)
    rng = np.random.default_rng(43)
    n3 = x.size
    nq = jq.size
    gx, gv = rng.standard_normal(n3), rng.standard_normal(n3)
    gjq, gjqd = rng.standard_normal(nq), rng.standard_normal(nq)
    E0 = np.asarray(d.youngs, np.float64).copy()
    nu0 = np.asarray(d.poisson, np.float64).copy()
    g = Scene(d)
    g.set_joint_state(jq, jqd)
    xg, vg = g.forward(x, v, n_steps=n, act=act)
    assert np.all(g.iterations(n) == d.max_iterations)
    jg, jdg = g.joint_state()
    grad = g.backward(gx, gv, gjq, gjqd)
    jg2, jdg2 = g.joint_state()  # the backward leaves the forward's final joint state
    assert np.array_equal(jg, jg2) and np.array_equal(jdg, jdg2)

    def loss(xx, vv, q, qd, aa, E):
        o.set_materials(E, nu0)
        o.set_joint_state(q, qd)
        r = o.forward(xx, vv, n_steps=n, act=aa)
        assert np.all(r["iters"] == d.max_iterations)
        q1, qd1 = o.joint_state()
        return gx @ r["x"] + gv @ r["v"] + gjq @ q1 + gjqd @ qd1

    base = dict(xx=x, vv=v, q=jq, qd=jqd, aa=act, E=E0)
    dirs = {
        "x": ("xx", 1e-3 * rng.standard_normal(n3)),
        "v": ("vv", 1e-2 * rng.standard_normal(n3)),
        "jq": ("q", 1e-3 * rng.standard_normal(nq)),
        "jqd": ("qd", 1e-3 * rng.standard_normal(nq)),
        "act": ("aa", 1e-2 * np.abs(act).max(initial=1.0) * rng.standard_normal(act.shape)),
        "E": ("E", 1e-3 * E0 * rng.standard_normal(E0.size)),
    }
    for key, (arg, dirn) in dirs.items():
        h = 1e-3
        lp = loss(**{**base, arg: base[arg] + h * dirn})
        lm = loss(**{**base, arg: base[arg] - h * dirn})
        fd = (lp - lm) / (2 * h)
        an = float(np.sum(np.asarray(grad[key]).reshape(-1) * dirn.reshape(-1)))
        assert abs(fd - an) <= 1e-5 * max(abs(fd), abs(an)) + 1e-9, (key, fd, an)
        assert abs(an) > 1e-6, (key, an)  # each direction moves the loss
    g.close()


def test_skeleton_adjoint_replays_and_checkpoints_are_identical():
    """With every step replayed from its checkpoint (no stored iterates) and
    with checkpoints every second step, the replays restart the links from
    each step's stored input joint state: the same gradients, bit for bit."""
    d, o, x, v, jq, jqd, act, n = _skeleton_case("articulated_beam")
    n = 5
    act = np.tile(act[:1], (n, 1))
    rng = np.random.default_rng(44)
    gx, gv = rng.standard_normal(x.size), rng.standard_normal(x.size)
    gjq, gjqd = rng.standard_normal(jq.size), rng.standard_normal(jq.size)
    out = []
    for every, budget in ((1, None), (1, 0), (2, None), (2, 0)):
        g = Scene(dataclasses.replace(d, checkpoint_every=every))
        if budget is not None:
            g.set_adjoint_budget(budget)
        g.set_joint_state(jq, jqd)
        g.forward(x, v, n_steps=n, act=act)
        out.append(g.backward(gx, gv, gjq, gjqd))
        g.close()
    for r in out[1:]:
        for key in ("x", "v", "E", "nu", "act", "jq", "jqd"):
            assert np.array_equal(out[0][key], r[key]), key
