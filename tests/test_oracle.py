"""Pins the CPU FP64 oracle (the checker) before anything is compared with it.

diff_fem ships no tests, golden vectors or output fixtures, and cannot be
built here, so the oracle is pinned by known-answer invariants of the
reference's algorithm (rest state, free fall, the projection's rules, the
kron structure of L, the soft-contact exchange's conservation laws) and by
central finite differences of the hand-written adjoint.  tests/golden/ holds
scene inputs in the reference's file formats (written by
tests/golden/make_fixtures.py), not oracle outputs.
"""
import dataclasses

import numpy as np
import pytest

from diff_fem_b200 import scene as S
from oracle import oracle as O

RNG = np.random.default_rng(42)


def rand_F(det_sign=1):
    while True:
        F = np.eye(3) + 0.4 * RNG.standard_normal((3, 3))
        if np.sign(np.linalg.det(F)) == det_sign and abs(np.linalg.det(F)) > 0.05:
            return F


def test_svd_reconstruction():
    for sign in (1, -1):
        for _ in range(20):
            F = rand_F(sign)
            U, s, V = O.svd3(F)
            assert np.allclose(U @ np.diag(s) @ V.T, F, atol=1e-13)
            assert np.allclose(U.T @ U, np.eye(3), atol=1e-13)
            assert np.allclose(V.T @ V, np.eye(3), atol=1e-13)
            assert np.all(s >= 0) and np.all(np.diff(s) <= 0)


def test_corotated_projection_rules():
    """md = polar rotation R (column 2 negated when det F < 0); md_volume has det +-1."""
    for sign in (1, -1):
        for _ in range(20):
            F = rand_F(sign)
            md, mdv = O.corot_project(F)
            U, s, Vt = np.linalg.svd(F)
            R = U @ Vt  # polar factor (numpy's SVD, independent of the oracle's)
            exp = R.copy()
            if np.linalg.det(F) < 0:
                exp[:, 2] *= -1
            assert np.allclose(md, exp, atol=1e-12)
            # volume projection: exactly 5 Newton steps on prod(S + D) = 1
            # (CorotateFEMConstraint.h:366-374), restated here with numpy
            D = np.zeros(3)
            for _ in range(5):
                p = s + D
                C = p.prod() - 1.0
                gr = np.array([p[1] * p[2], p[0] * p[2], p[0] * p[1]])
                D = (gr @ D - C) / (gr @ gr) * gr
            assert np.allclose(mdv, U @ np.diag(s + D) @ Vt, atol=1e-12)
            assert np.sign(np.linalg.det(mdv)) == np.sign(np.linalg.det(F))


def test_corotated_vjp_matches_finite_differences():
    for sign in (1, -1):
        for _ in range(10):
            F = rand_F(sign)
            gmd = RNG.standard_normal((3, 3))
            gmdv = RNG.standard_normal((3, 3))
            gF = O.corot_vjp(F, gmd, gmdv)
            dF = RNG.standard_normal((3, 3))
            eps = 1e-6
            mp, vp = O.corot_project(F + eps * dF)
            mm, vm = O.corot_project(F - eps * dF)
            fd = (np.sum(gmd * (mp - mm)) + np.sum(gmdv * (vp - vm))) / (2 * eps)
            assert abs(np.sum(gF * dF) - fd) < 1e-7 * max(1.0, abs(fd))


def test_vjp_equal_singular_values():
    """Exact divided differences: no blow-up for repeated singular values."""
    Q, _ = np.linalg.qr(RNG.standard_normal((3, 3)))
    for F in (np.eye(3) * 1.1, Q @ np.diag([1.2, 1.2, 0.9]) @ Q.T):
        g = O.corot_vjp(F, RNG.standard_normal((3, 3)), RNG.standard_normal((3, 3)))
        assert np.all(np.isfinite(g))


def test_ccd_known_answers():
    """Vertex-face CCD against a static triangle in the y = 0 plane."""
    tri = ([0, 0, 0], [1, 0, 1], [1, 0, 0])
    hit, n = O.vf_impact([0.2, 0.1, 0.2], [0.2, -0.1, 0.2], *tri)       # crossing
    assert hit and abs(abs(n[1]) - np.sin(np.pi / 4)) < 1e-12
    assert not O.vf_impact([0.2, 0.1, 0.2], [0.3, 0.1, 0.2], *tri)[0]  # parallel, above
    assert O.vf_impact([0.2, 0.1, 0.2], [0.2, 5e-5, 0.2], *tri)[0]     # ends within the thickness
    assert not O.vf_impact([0.2, 0.1, 0.2], [0.2, 2e-4, 0.2], *tri)[0] # ends outside the thickness
    assert not O.vf_impact([2, 0.1, 0.2], [2, -0.1, 0.2], *tri)[0]     # misses the face
    assert O.vf_impact([1.00005, 0.1, 0.5], [1.00005, -0.1, 0.5], *tri)[0] is False  # outside edge, crossing
    assert O.vf_impact([1.00005, 0.1, 0.5], [1.00005, 0.00005, 0.5], *tri)[0]       # near the edge at t = 1


def test_contact_keeps_the_body_above_the_ground():
    d = S.drop_box()
    o = O.OracleScene(d)
    r = o.forward(d.x0.reshape(-1).copy(), d.initial_velocity.copy(), n_steps=40, traj=True)
    assert o.contact_passes().sum() > 0
    assert r["traj"].reshape(40, -1, 3)[:, :, 1].min() > -1e-3
    # the same box without contact falls through
    d.handle_collision = False
    o2 = O.OracleScene(d)
    r2 = o2.forward(d.x0.reshape(-1).copy(), d.initial_velocity.copy(), n_steps=40, traj=True)
    assert r2["traj"].reshape(40, -1, 3)[:, :, 1].min() < -0.1


def test_lumped_masses_match_builder():
    d = S.cantilever()
    m = O.lumped_masses(d.x0, d.tets, 20.0, True)
    assert np.allclose(m, d.mass, rtol=1e-14)
    m2 = O.lumped_masses(d.x0, d.tets, 20.0, False)
    assert np.allclose(m2, 20.0 / d.n_vertices)


def test_kron_structure_of_L():
    """The reference's 3N x 3N L (per-constraint A_i^T A_i triplets) equals kron(L_s, I3)."""
    for d in (S.cantilever(), S.muscle_beam(), S.cloth_sheet(nv=5)):
        d.bend_weight = d.bend_weight * 0  # bending enters Hs only; checked via Hs below
        o = O.OracleScene(d)
        N = d.n_vertices
        r, c, v = o.full_L_triplets()
        L3 = np.zeros((3 * N, 3 * N))
        np.add.at(L3, (r, c), v)
        hr, hc, hv = o.hs_coo()
        Hs = np.zeros((N, N))
        np.add.at(Hs, (hr, hc), hv)
        Ls = Hs - np.diag(d.mass / d.time_step ** 2)
        assert np.allclose(L3, np.kron(Ls, np.eye(3)), rtol=1e-12, atol=1e-9 * np.abs(Ls).max())


def test_rest_state_is_a_fixed_point():
    """No gravity, zero velocity, rest positions: every projection reproduces the
    rest configuration, so the state stays put."""
    for d in (S.cantilever(), S.muscle_beam(), S.cloth_sheet(nv=6)):
        d.gravity = (0.0, 0.0, 0.0)
        o = O.OracleScene(d)
        x = d.x0.reshape(-1).copy()
        r = o.forward(x, np.zeros_like(x), n_steps=3)
        assert np.abs(r["x"] - x).max() < 1e-9 * max(1.0, np.abs(x).max())


def test_free_fall_is_exact():
    """Unpinned body in its rest shape: x' = x + h (v + g h), v' = damping (v + g h)."""
    d = S.cantilever()
    d.attach_vertex = np.zeros(0, np.int32)
    d.attach_target = np.zeros((0, 3))
    d.attach_stiffness = np.zeros(0)
    o = O.OracleScene(d)
    x = d.x0.reshape(-1).copy()
    v = np.tile([0.3, 0.1, -0.2], d.n_vertices)
    r = o.forward(x, v, n_steps=1)
    g = np.tile(d.gravity, d.n_vertices)
    vwc = v + g * d.time_step
    assert np.allclose(r["x"], x + d.time_step * vwc, atol=1e-10)
    assert np.allclose(r["v"], d.damping * vwc, atol=1e-8)


def test_deterministic():
    d = S.muscle_beam()
    o = O.OracleScene(d)
    x = d.x0.reshape(-1).copy()
    act = RNG.uniform(0, 1, (4, d.n_segments))
    a = o.forward(x, np.zeros_like(x), n_steps=4, act=act)
    b = o.forward(x, np.zeros_like(x), n_steps=4, act=act)
    assert np.array_equal(a["x"], b["x"]) and np.array_equal(a["v"], b["v"])


def test_multithreaded_local_step_is_identical():
    d = S.inverse_stiffness(nx=8, ny=4, nz=4)
    o = O.OracleScene(d)
    x = d.x0.reshape(-1).copy()
    a = o.forward(x, np.zeros_like(x), n_steps=2, threads=1)
    b = o.forward(x, np.zeros_like(x), n_steps=2, threads=4)
    assert np.array_equal(a["x"], b["x"])


def _loss(o, x, v, gx, gv, n, act=None):
    r = o.forward(x, v, n_steps=n, act=act)
    return gx @ r["x"] + gv @ r["v"], r["iters"]


@pytest.mark.parametrize("builder", ["cantilever", "muscle_beam", "cloth_sheet", "pneumatic_beam"])
def test_adjoint_matches_central_differences(builder):
    """Each case draws from its own seed (the check needs iteration counts
    that no perturbation changes, a property of the draw, so the draw must
    not depend on which tests ran before)."""
    d = getattr(S, builder)()
    o = O.OracleScene(d)
    n = 3
    rng = np.random.default_rng({"cantilever": 101, "muscle_beam": 102, "cloth_sheet": 103, "pneumatic_beam": 104}[builder])
    x = d.x0.reshape(-1) + 1e-3 * rng.standard_normal(3 * d.n_vertices)
    v = 0.05 * rng.standard_normal(3 * d.n_vertices)
    gx = rng.standard_normal(x.size)
    gv = rng.standard_normal(x.size)
    act = rng.uniform(0, 1, (n, d.n_segments)) if d.n_segments else None
    _, it0 = _loss(o, x, v, gx, gv, n, act)
    g = o.backward(gx, gv)
    checks = []
    dx = rng.standard_normal(x.size)
    eps = 1e-6
    (lp, ip), (lm, im) = _loss(o, x + eps * dx, v, gx, gv, n, act), _loss(o, x - eps * dx, v, gx, gv, n, act)
    checks.append((g["x"] @ dx, (lp - lm) / (2 * eps), ip, im))
    dv = rng.standard_normal(x.size)
    (lp, ip), (lm, im) = _loss(o, x, v + eps * dv, gx, gv, n, act), _loss(o, x, v - eps * dv, gx, gv, n, act)
    checks.append((g["v"] @ dv, (lp - lm) / (2 * eps), ip, im))
    if d.n_tets:
        E, nu = d.youngs.copy(), d.poisson.copy()
        dE = rng.standard_normal(E.size) * E
        rel = 1e-5
        o.set_materials(E + rel * dE, nu); lp, ip = _loss(o, x, v, gx, gv, n, act)
        o.set_materials(E - rel * dE, nu); lm, im = _loss(o, x, v, gx, gv, n, act)
        o.set_materials(E, nu)
        checks.append((g["E"] @ dE, (lp - lm) / (2 * rel), ip, im))
    if act is not None:
        da = rng.standard_normal(act.shape)
        (lp, ip), (lm, im) = _loss(o, x, v, gx, gv, n, act + eps * da), _loss(o, x, v, gx, gv, n, act - eps * da)
        checks.append((np.sum(g["act"] * da), (lp - lm) / (2 * eps), ip, im))
    for adj, fd, ip, im in checks:
        assert np.array_equal(ip, it0) and np.array_equal(im, it0), "iteration count changed under perturbation"
        assert abs(adj - fd) <= 1e-5 * max(1.0, abs(fd)), (adj, fd)


@pytest.mark.parametrize("case", ["drop", "slide"])
def test_contact_adjoint_matches_central_differences(case):
    """The contact phase's reverse (Jacobi sweeps, friction cone, relaxation)
    against central differences, on a box that lands on the ground during
    the window (impacts and normals are constants of the tape); "slide" lands
    with a tangential velocity, so the friction cone clamps."""
    d = S.drop_box(mu=0.3)
    o = O.OracleScene(d)
    n = 3 if case == "drop" else 4
    rng = np.random.default_rng(11)
    x = d.x0.reshape(-1).copy()
    v = d.initial_velocity.copy() if case == "drop" else np.tile([1.0, -1.0, 0.3], d.n_vertices)
    gx, gv = rng.standard_normal(x.size), rng.standard_normal(x.size)
    _, it0 = _loss(o, x, v, gx, gv, n)
    p0 = o.contact_passes()
    assert p0.sum() > 0
    g = o.backward(gx, gv)
    eps = 1e-7
    checks = []
    for name in ("x", "v", "E"):
        if name == "E":
            E, nu = d.youngs.copy(), d.poisson.copy()
            dE = rng.standard_normal(E.size) * E
            o.set_materials(E + eps * dE, nu); lp, ip = _loss(o, x, v, gx, gv, n); pp = o.contact_passes()
            o.set_materials(E - eps * dE, nu); lm, im = _loss(o, x, v, gx, gv, n); pm = o.contact_passes()
            o.set_materials(E, nu)
            checks.append((g["E"] @ dE, (lp - lm) / (2 * eps), ip, im, pp, pm))
            continue
        dz = rng.standard_normal(x.size)
        if name == "x":
            (lp, ip), pp = _loss(o, x + eps * dz, v, gx, gv, n), o.contact_passes()
            (lm, im), pm = _loss(o, x - eps * dz, v, gx, gv, n), o.contact_passes()
        else:
            (lp, ip), pp = _loss(o, x, v + eps * dz, gx, gv, n), o.contact_passes()
            (lm, im), pm = _loss(o, x, v - eps * dz, gx, gv, n), o.contact_passes()
        checks.append((g[name] @ dz, (lp - lm) / (2 * eps), ip, im, pp, pm))
    for adj, fd, ip, im, pp, pm in checks:
        assert np.array_equal(ip, it0) and np.array_equal(im, it0)
        assert np.array_equal(pp, p0) and np.array_equal(pm, p0)
        assert abs(adj - fd) <= 1e-4 * max(1.0, abs(fd)), (adj, fd)


def test_underwater_drag_forces_and_adjoint():
    """Underwater drag and lift (Dfobj::ComputeDragForces): a block swimming
    through still water slows down (drag opposes the motion; no gravity
    underwater), and the adjoint through the per-face forces matches central
    differences in x and v."""
    d, v0 = S.underwater_block()
    o = O.OracleScene(d)
    x = d.x0.reshape(-1).copy()
    v = v0.reshape(-1).copy()
    r = o.forward(x, v, n_steps=4)
    mom0 = (d.mass[:, None] * v0).sum(0)
    mom1 = (d.mass[:, None] * r["v"].reshape(-1, 3)).sum(0)
    assert np.dot(mom1, mom0) < 0.999 * np.dot(mom0, mom0)        # water took momentum
    dry = O.OracleScene(dataclasses.replace(d, drag_faces=np.zeros((0, 3), np.int32)))
    rd = dry.forward(x, v, n_steps=4)
    # no gravity underwater: without the drag faces the mass-weighted vertical
    # velocity stays put (gravity would add 9.8 * 4/60 = 0.65 m/s)
    vy0 = (d.mass * v0[:, 1]).sum() / d.mass.sum()
    vy1 = (d.mass * rd["v"].reshape(-1, 3)[:, 1]).sum() / d.mass.sum()
    assert abs(vy1 - vy0) < 0.01
    rng = np.random.default_rng(21)
    n = 3
    gx, gv = rng.standard_normal(x.size), rng.standard_normal(x.size)
    _, it0 = _loss(o, x, v, gx, gv, n)
    g = o.backward(gx, gv)
    eps = 1e-6
    for name in ("x", "v"):
        dz = rng.standard_normal(x.size)
        if name == "x":
            (lp, ip), (lm, im) = _loss(o, x + eps * dz, v, gx, gv, n), _loss(o, x - eps * dz, v, gx, gv, n)
        else:
            (lp, ip), (lm, im) = _loss(o, x, v + eps * dz, gx, gv, n), _loss(o, x, v - eps * dz, gx, gv, n)
        assert np.array_equal(ip, it0) and np.array_equal(im, it0)
        fd = (lp - lm) / (2 * eps)
        assert abs(g[name] @ dz - fd) <= 1e-5 * max(1.0, abs(fd)), (name, g[name] @ dz, fd)


def test_self_group_exchange_invariants():
    """One soft-contact face group (World.h:1462-1531): the normal self
    forces sum to zero; the face's vertices end with one common velocity;
    every approaching group vertex ends with the face's normal velocity; a
    receding one is left alone; with a large friction coefficient every
    member sticks (common full velocity) and the full self forces sum to
    zero.  (With sliding members the reference's friction does not balance:
    the sticking set receives mu f_n along the mean slip, each sliding
    vertex mu r_n m_k / (m_k + m_stick) along its own slip; its sanity
    assert in do_solve_friction is compiled out.)"""
    rng = np.random.default_rng(17)
    for trial in range(20):
        k = int(rng.integers(1, 6))
        nrm = rng.standard_normal(3)
        P = rng.standard_normal((3 + k, 3))
        m = rng.uniform(0.5, 2.0, 3 + k)
        mu = 1e9 if trial % 2 else 0.3
        out, inc = O.self_group(nrm, P, m, mu)
        scale = np.abs(P).max()
        n = nrm / np.linalg.norm(nrm)
        assert abs(out.sum(0) @ n) <= 1e-12 * scale * (3 + k)
        if mu > 1e6:
            assert np.abs(out.sum(0)).max() <= 1e-12 * scale * (3 + k)
        vel = (P + out) / m[:, None]
        assert np.allclose(vel[0], vel[1], atol=1e-12 * scale) and np.allclose(vel[0], vel[2], atol=1e-12 * scale)
        face_vn = (P[:3].sum(0) @ n) / m[:3].sum()
        for q in range(k):
            rel = (P[3 + q] @ n) / m[3 + q] - face_vn
            assert inc[q] == (rel <= 0)
            if inc[q]:
                assert abs(vel[3 + q] @ n - vel[0] @ n) <= 1e-10 * max(1.0, scale)
                if mu > 1e6:
                    assert np.allclose(vel[3 + q], vel[0], atol=1e-10 * max(1.0, scale))
            else:
                assert np.all(out[3 + q] == 0)


def test_soft_contact_keeps_the_cloth_on_the_block():
    """Self-collision on: a cloth dropped onto a soft block (both are soft
    contact surfaces) stays above the block's top; with it off the cloth
    falls through the block."""
    d = S.cloth_on_block()
    nc = 16
    x = d.x0.reshape(-1).copy()
    v = d.initial_velocity.copy()
    o = O.OracleScene(d)
    r = o.forward(x, v, n_steps=8, traj=True)
    tr = r["traj"].reshape(8, -1, 3)
    assert o.contact_passes().sum() > 0
    for s in range(8):
        assert tr[s, :nc, 1].min() > tr[s, nc:, 1].max()
    off = O.OracleScene(dataclasses.replace(d, self_collision=False))
    tr2 = off.forward(x, v, n_steps=8, traj=True)["traj"].reshape(8, -1, 3)
    assert tr2[:, :nc, 1].min() < 0.02


def test_soft_contact_steps_carry_no_remembered_forces():
    """Every time step starts with zero remembered contact forces
    (World::TimeStepping -> updateCollisionScene, World.h:700,742-753), so a
    2-step forward equals two 1-step forwards bit for bit."""
    d = S.cloth_on_block()
    x = d.x0.reshape(-1).copy()
    v = d.initial_velocity.copy()
    o = O.OracleScene(d)
    r2 = o.forward(x, v, n_steps=2)
    assert o.contact_passes().sum() > 0
    r1 = o.forward(x, v, n_steps=1)
    r1b = o.forward(r1["x"], r1["v"], n_steps=1)
    assert np.array_equal(r2["x"], r1b["x"]) and np.array_equal(r2["v"], r1b["v"])


def test_soft_contact_adjoint_matches_central_differences():
    """The soft-contact adjoint (face groups by forward-mode duals, the
    self-force state carried between the Jacobi iterations of a step) against
    central differences.  The detection's outputs (normals from the faces'
    start positions, groups) are constants of the tape, as on the
    reference's tape, so the perturbed runs replay the recorded detection."""
    d = S.cloth_on_block()
    o = O.OracleScene(d)
    n = 3
    rng = np.random.default_rng(5)
    x = d.x0.reshape(-1).copy()
    v = d.initial_velocity.copy()
    gx, gv = rng.standard_normal(x.size), rng.standard_normal(x.size)
    o.detection_replay(1)
    _, it0 = _loss(o, x, v, gx, gv, n)
    assert o.contact_passes().sum() >= n
    g = o.backward(gx, gv)
    o.detection_replay(2)
    eps = 1e-7
    E, nu = d.youngs.copy(), d.poisson.copy()
    dE = rng.standard_normal(E.size) * E
    o.set_materials(E + eps * dE, nu); lp, ip = _loss(o, x, v, gx, gv, n)
    o.set_materials(E - eps * dE, nu); lm, im = _loss(o, x, v, gx, gv, n)
    o.set_materials(E, nu)
    checks = [(g["E"] @ dE, (lp - lm) / (2 * eps), ip, im)]
    for name in ("x", "v"):
        dz = rng.standard_normal(x.size)
        if name == "x":
            (lp, ip), (lm, im) = _loss(o, x + eps * dz, v, gx, gv, n), _loss(o, x - eps * dz, v, gx, gv, n)
        else:
            (lp, ip), (lm, im) = _loss(o, x, v + eps * dz, gx, gv, n), _loss(o, x, v - eps * dz, gx, gv, n)
        checks.append((g[name] @ dz, (lp - lm) / (2 * eps), ip, im))
    for adj, fd, ip, im in checks:
        assert np.array_equal(ip, it0) and np.array_equal(im, it0)
        assert abs(adj - fd) <= 1e-5 * max(1.0, abs(fd)), (adj, fd)


# ---- articulated skeleton (Link, sim/constants.h; World::ComputeSolution's rigid branch)

def _damped_fall(h, g, damping, n):
    """Centre-of-mass displacement of n damped free-fall steps from rest:
    x_{k+1} = x_k + h v_k + h^2 g, v_{k+1} = damping (x_{k+1} - x_k) / h."""
    x, v = 0.0, 0.0
    for _ in range(n):
        dx = h * v + h * h * g
        x += dx
        v = damping * dx / h
    return x


def test_skeleton_rest_state_is_a_fixed_point():
    d = S.articulated_beam(gravity=(0.0, 0.0, 0.0))
    o = O.OracleScene(d)
    x = d.x0.reshape(-1).copy()
    r = o.forward(x, np.zeros_like(x), n_steps=3)
    jq, jqd = o.joint_state()
    assert np.abs(r["x"] - x).max() < 1e-14
    eye = np.r_[np.eye(3).reshape(-1), np.zeros(3 + 2)]
    assert np.abs(jq - eye).max() < 1e-14 and np.abs(jqd - eye).max() < 1e-14


def test_skeleton_links_stay_rigid_and_the_centre_of_mass_falls_freely():
    """Each link's vertices keep their rest distances (V0 = prefix Tr (rest -
    joint) with rotations); the centre of mass follows damped free fall (the
    link system's root-translation rows make the reaction on the rigid
    vertices sum to zero; what remains is the second-order gap between the
    linearised link update the solve assumed and UpdateT's)."""
    d = S.articulated_beam()
    o = O.OracleScene(d)
    n = 6
    x = d.x0.reshape(-1).copy()
    act = np.tile([0.5, 2.0], (n, 1))
    r = o.forward(x, np.zeros_like(x), n_steps=n, act=act)
    X, X0 = r["x"].reshape(-1, 3), x.reshape(-1, 3)
    for l in range(3):
        vs = d.link_vertices[d.link_offsets[l]:d.link_offsets[l + 1]]
        D = np.linalg.norm(X[vs][:, None] - X[vs][None], axis=2)
        D0 = np.linalg.norm(X0[vs][:, None] - X0[vs][None], axis=2)
        assert np.abs(D - D0).max() < 1e-13, l
    m = d.mass
    com = (m[:, None] * (X - X0)).sum(0) / m.sum()
    fall = _damped_fall(d.time_step, -9.8, d.damping, n)
    assert abs(com[1] - fall) < 1e-6 * abs(fall) and abs(com[0]) < 1e-6 * abs(fall) and abs(com[2]) < 1e-12
    jq, jqd = o.joint_state()
    assert jq.size == 14 and abs(jq[12]) > 1e-3 and abs(jq[13]) > 1e-4  # the torques turned / slid the links
    R = jq[:9].reshape(3, 3)
    assert abs(np.linalg.det(R) - 1.0) < 1e-3  # T.R = (I + [w]x) Tr.R: a rotation to first order


def test_skeleton_joint_state_round_trip_and_determinism():
    d = S.articulated_beam()
    x = d.x0.reshape(-1).copy()
    act = np.tile([0.5, 2.0], (4, 1))
    a = O.OracleScene(d)
    ra = a.forward(x, np.zeros_like(x), n_steps=4, act=act)
    b = O.OracleScene(d)
    rb1 = b.forward(x, np.zeros_like(x), n_steps=2, act=act[:2])
    jq, jqd = b.joint_state()
    c = O.OracleScene(d)
    c.set_joint_state(jq, jqd)
    rc = c.forward(rb1["x"], rb1["v"], n_steps=2, act=act[2:])
    assert np.array_equal(rc["x"], ra["x"]) and np.array_equal(c.joint_state()[0], a.joint_state()[0])
