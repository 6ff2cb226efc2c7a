"""Batches of independent scenes (dfem_scene_create_batch) against the same
scenes stepped one at a time.

Every part of a batch runs the same arithmetic in the same order as the scene
alone (its own convergence test, iteration count and factor; part-aligned
reduction blocks), so positions, velocities, iteration counts and gradients
must agree bit for bit.
"""
import dataclasses

import numpy as np
import pytest

from diff_fem_b200 import _capi, scene as S
from diff_fem_b200.engine import Scene

pytestmark = pytest.mark.gpu



def one_scene(d):
    """A single scene in a triangular-solve form: a batch's solves run the
    same per-supernode arithmetic, so the two agree bit for bit (the dense
    inverse form the autotune may pick for a small single scene agrees to
    rounding only)."""
    s = Scene(d)
    if s.solve_mode()["mode"] == "dense":
        s.solve_mode("persistent")
    return s

def harmonise(descs, precision=_capi.DFEM_PREC_FP64):
    """Batch members share time step, iteration cap, damping and gravity."""
    return [dataclasses.replace(d, time_step=1.0 / 60.0, max_iterations=15, damping=0.9999,
                                gravity=(0.0, -9.8, 0.0), precision=precision) for d in descs]


def mixed_scenes(precision=_capi.DFEM_PREC_FP64):
    return harmonise([S.inverse_stiffness(nx=10, ny=3, nz=3), S.muscle_beam(), S.cantilever(),
                      S.cloth_sheet(nv=8), S.inverse_stiffness(nx=6, ny=2, nz=2, seed=7)], precision)


def concat_state(descs):
    x = np.concatenate([d.x0.reshape(-1) for d in descs])
    return x, np.zeros_like(x)


def split(a, offs, scale=3):
    return [a[scale * offs[i]: scale * offs[i + 1]] for i in range(len(offs) - 1)]


@pytest.mark.parametrize("precision", [_capi.DFEM_PREC_FP64, _capi.DFEM_PREC_MIXED])
def test_batch_matches_scenes_one_at_a_time(precision):
    descs = mixed_scenes(precision)
    n = 6
    b = Scene.batch(descs)
    assert b.nparts == len(descs)
    vo = b.offsets["vertices"]
    assert list(np.diff(vo)) == [d.n_vertices for d in descs]
    nseg = [d.n_segments for d in descs]
    rng = np.random.default_rng(3)
    acts = [rng.uniform(0, 1, (n, k)) for k in nseg]
    act = np.concatenate(acts, axis=1) if sum(nseg) else None
    x, v = concat_state(descs)
    xb, vb, tb = b.forward(x, v, n_steps=n, act=act, traj=True)
    itb = b.iterations(n)
    assert itb.shape == (n, len(descs))
    gx = rng.standard_normal(x.size)
    gv = rng.standard_normal(x.size)
    gb = b.backward(gx, gv)
    to = b.offsets["tets"]
    so = b.offsets["segments"]
    for p, d in enumerate(descs):
        s = one_scene(d)
        xs, vs, ts = s.forward(d.x0.reshape(-1), np.zeros(3 * d.n_vertices), n_steps=n,
                               act=acts[p] if nseg[p] else None, traj=True)
        assert np.array_equal(s.iterations(n), itb[:, p]), p
        assert np.array_equal(split(xb, vo)[p], xs), p
        assert np.array_equal(split(vb, vo)[p], vs), p
        assert np.array_equal(tb[:, 3 * vo[p]: 3 * vo[p + 1]], ts), p
        gs = s.backward(split(gx, vo)[p], split(gv, vo)[p])
        assert np.array_equal(split(gb["x"], vo)[p], gs["x"]), p
        assert np.array_equal(split(gb["v"], vo)[p], gs["v"]), p
        assert np.array_equal(gb["E"][to[p]:to[p + 1]], gs["E"]), p
        assert np.array_equal(gb["nu"][to[p]:to[p + 1]], gs["nu"]), p
        if nseg[p]:
            assert np.array_equal(gb["act"][:, so[p]:so[p + 1]], gs["act"]), p
        s.close()
    b.close()


@pytest.mark.parametrize("precision,every", [(_capi.DFEM_PREC_FP64, 1), (_capi.DFEM_PREC_MIXED, 1),
                                             (_capi.DFEM_PREC_MIXED, 3)])
def test_batch_with_underwater_parts_matches_scenes(precision, every):
    """Underwater parts (drag and lift on their faces, no gravity) batched
    with dry ones: each part's trajectory, iteration counts and gradients are
    the scene's own, bit for bit, with checkpoints every step or every third
    (the adjoint then regenerates the segments' drag inputs)."""
    (wa, va), (wb, vb_) = S.underwater_block(), S.underwater_block(nx=3, ny=3, nz=2, speed=0.9, seed=5)
    dry = S.muscle_beam()
    descs = [dataclasses.replace(d, checkpoint_every=every)
             for d in harmonise([wa, dry, wb], precision)]
    vels = [va.reshape(-1), np.tile([0.2, 0.1, -0.3], dry.n_vertices), vb_.reshape(-1)]
    n = 5
    b = Scene.batch(descs)
    vo, to, so = b.offsets["vertices"], b.offsets["tets"], b.offsets["segments"]
    nseg = [d.n_segments for d in descs]
    rng = np.random.default_rng(11)
    acts = [rng.uniform(0, 1, (n, k)) for k in nseg]
    x = np.concatenate([d.x0.reshape(-1) for d in descs])
    v = np.concatenate(vels)
    xb, vb, tb = b.forward(x, v, n_steps=n, act=np.concatenate(acts, axis=1), traj=True)
    itb = b.iterations(n)
    gx, gv = rng.standard_normal(x.size), rng.standard_normal(x.size)
    gb = b.backward(gx, gv)
    for p, d in enumerate(descs):
        s = one_scene(d)
        xs, vs, ts = s.forward(d.x0.reshape(-1), vels[p], n_steps=n, act=acts[p] if nseg[p] else None, traj=True)
        assert np.array_equal(s.iterations(n), itb[:, p]), p
        assert np.array_equal(split(xb, vo)[p], xs), p
        assert np.array_equal(split(vb, vo)[p], vs), p
        assert np.array_equal(tb[:, 3 * vo[p]: 3 * vo[p + 1]], ts), p
        gs = s.backward(split(gx, vo)[p], split(gv, vo)[p])
        for k in ("x", "v"):
            assert np.array_equal(split(gb[k], vo)[p], gs[k]), (p, k)
        for k in ("E", "nu"):
            assert np.array_equal(gb[k][to[p]:to[p + 1]], gs[k]), (p, k)
        if nseg[p]:
            assert np.array_equal(gb["act"][:, so[p]:so[p + 1]], gs["act"]), p
        s.close()
    b.close()


def test_batch_set_materials_refactors_each_part():
    descs = harmonise([S.inverse_stiffness(nx=8, ny=3, nz=3, seed=s) for s in (1, 2, 3)])
    b = Scene.batch(descs)
    E = np.concatenate([S.log_uniform_moduli(d.n_tets, 100 + i) for i, d in enumerate(descs)])
    nu = np.full(E.size, 0.3)
    b.set_materials(E, nu)
    x, v = concat_state(descs)
    xb, _ = b.forward(x, v, n_steps=4)
    vo, to = b.offsets["vertices"], b.offsets["tets"]
    for p, d in enumerate(descs):
        s = one_scene(d)
        s.set_materials(E[to[p]:to[p + 1]], nu[to[p]:to[p + 1]])
        xs, _ = s.forward(d.x0.reshape(-1), np.zeros(3 * d.n_vertices), n_steps=4)
        assert np.array_equal(split(xb, vo)[p], xs)
        s.close()
    b.close()


def test_batch_rejects_soft_contact():
    d = dataclasses.replace(S.cloth_on_block(), obstacle_x=np.zeros((0, 3)), obstacle_faces=np.zeros((0, 3), np.int32))
    with pytest.raises(_capi.DfemError, match="soft-soft"):
        Scene.batch([d, d])


def test_batch_rejects_mismatched_time_steps():
    descs = [S.cantilever(), S.inverse_stiffness(nx=6, ny=2, nz=2)]
    with pytest.raises(_capi.DfemError, match="time_step"):
        Scene.batch(descs)


@pytest.mark.parametrize("form", ["auto", "levels", "split"])
def test_large_batch_launch_classes_match_scenes(form):
    """A batch of many supernodes: launch classes per level (one supernode per
    warp, small and large CTAs), the split and tail-selected solve forms; each
    scene alone runs its own factor's schedule and form.  Neither moves any
    arithmetic: bit-identical."""
    descs, _ = S.uneven_batch(n_scenes=32, t_hi=1e4, precision=_capi.DFEM_PREC_FP64, ground=False)
    b = Scene.batch(descs)
    assert b.info()["n_supernodes"] > 2048
    info = b.solve_mode(form)
    if form != "auto":
        assert info["mode"] == form
    n = 2
    x, v = concat_state(descs)
    xb, vb = b.forward(x, v, n_steps=n)
    rng = np.random.default_rng(4)
    gx = rng.standard_normal(x.size)
    gb = b.backward(gx, np.zeros_like(gx))
    vo, to = b.offsets["vertices"], b.offsets["tets"]
    itb = b.iterations(n)
    for p in range(0, len(descs), 5):
        d = descs[p]
        s = one_scene(d)
        xs, vs = s.forward(d.x0.reshape(-1), np.zeros(3 * d.n_vertices), n_steps=n)
        assert np.array_equal(s.iterations(n), itb[:, p]), p
        assert np.array_equal(split(xb, vo)[p], xs), p
        assert np.array_equal(split(vb, vo)[p], vs), p
        gs = s.backward(split(gx, vo)[p], np.zeros(3 * d.n_vertices))
        assert np.array_equal(split(gb["x"], vo)[p], gs["x"]), p
        assert np.array_equal(gb["E"][to[p]:to[p + 1]], gs["E"]), p
        s.close()
    b.close()


@pytest.mark.parametrize("form", ["loop", "cooperative"])
def test_batch_with_obstacle_contact_matches_scenes(form):
    """Obstacle contact inside a batch: boxes dropped on their own grounds (one
    with friction clamping, one landing faster) and a muscle beam without
    contact.  The contact parts' trajectories, contact passes, iteration
    counts and gradients are the scene's own bit for bit (each part runs its
    own detection passes, Jacobi iterations and convergence test, as a loop
    of gated kernels or in one cooperative launch); the part without contact
    matches to rounding (its adjoint passes through the phase's cotangent
    bookkeeping)."""
    a = S.drop_box(mu=0.3)
    b_ = S.drop_box(nx=3, ny=2, nz=3, height=0.03, v0=-1.5, mu=0.3)
    dry = S.muscle_beam()
    descs = harmonise([a, b_, dry])
    vels = [a.initial_velocity, b_.initial_velocity, np.zeros(3 * dry.n_vertices)]
    n = 8
    bt = Scene.batch(descs)
    bt.set_option("fused_contact", 1 if form == "cooperative" else 0)
    vo, to, so = bt.offsets["vertices"], bt.offsets["tets"], bt.offsets["segments"]
    nseg = [d.n_segments for d in descs]
    rng = np.random.default_rng(17)
    acts = [rng.uniform(0, 1, (n, k)) for k in nseg]
    x = np.concatenate([d.x0.reshape(-1) for d in descs])
    v = np.concatenate(vels)
    xb, vb, tb = bt.forward(x, v, n_steps=n, act=np.concatenate(acts, axis=1), traj=True)
    itb = bt.iterations(n)
    passes_b = bt.contact_passes(n)
    gx, gv = rng.standard_normal(x.size), rng.standard_normal(x.size)
    gb = bt.backward(gx, gv)
    passes = []
    for p, d in enumerate(descs):
        s = one_scene(d)
        xs, vs, ts = s.forward(d.x0.reshape(-1), vels[p], n_steps=n, act=acts[p] if nseg[p] else None, traj=True)
        assert np.array_equal(s.iterations(n), itb[:, p]), p
        assert np.array_equal(split(xb, vo)[p], xs), p
        assert np.array_equal(split(vb, vo)[p], vs), p
        assert np.array_equal(tb[:, 3 * vo[p]: 3 * vo[p + 1]], ts), p
        gs = s.backward(split(gx, vo)[p], split(gv, vo)[p])
        contact = p < 2
        if contact:
            passes.append(s.contact_passes(n))
            assert passes[-1].sum() > 0, p
        for k in ("x", "v"):
            if contact:
                assert np.array_equal(split(gb[k], vo)[p], gs[k]), (p, k)
            else:
                assert np.allclose(split(gb[k], vo)[p], gs[k], rtol=1e-12, atol=1e-12 * np.abs(gs[k]).max()), (p, k)
        for k in ("E", "nu"):
            if contact:
                assert np.array_equal(gb[k][to[p]:to[p + 1]], gs[k]), (p, k)
            else:
                assert np.allclose(gb[k][to[p]:to[p + 1]], gs[k], rtol=1e-12, atol=1e-12 * np.abs(gs[k]).max()), (p, k)
        if nseg[p]:
            assert np.allclose(gb["act"][:, so[p]:so[p + 1]], gs["act"], rtol=1e-12,
                               atol=1e-12 * np.abs(gs["act"]).max()), p
        s.close()
    assert np.array_equal(passes_b, np.maximum(passes[0], passes[1]))  # a batch reports its parts' most passes
    bt.close()
