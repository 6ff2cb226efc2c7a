"""The allocation-free corotated local step (dfem_eval_corotated_noalloc).

Some callers cannot allocate device memory (a pool that owns the whole device
heap, a runtime that may only pass pre-allocated buffers).  For them the
library offers a variant of the local-step kernel whose scratch is a static
device array; the caller passes inputs and outputs.  This test calls it
through the C ABI on device buffers it owns and checks it against the
allocating path (dfem_eval_local of a scene with the same tets), within the
tolerance of the other parity tests, on two calls in a row.  It lives in a
file of its own that pytest collects last, and it works both alone in a fresh
process (the first call looks up the scratch's device address) and after the
other tests.
"""
import numpy as np
import pytest

from diff_fem_b200 import _capi, scene as S
from diff_fem_b200.engine import Scene

pytestmark = pytest.mark.gpu

TOL = 1e-9


def raw_arrays(d):
    """Re-oriented tets, row-major invDm, weights and the vertex incidence CSR,
    built here in numpy the way the reference sets a tet up (Dfobj.h:474-503)."""
    x0 = d.x0.reshape(-1, 3)
    tets = d.tets.reshape(-1, 4).astype(np.int32).copy()
    Dm = np.stack([x0[tets[:, k]] - x0[tets[:, 0]] for k in (1, 2, 3)], axis=2)
    neg = np.linalg.det(Dm) < 0
    tets[neg, 1], tets[neg, 2] = tets[neg, 2].copy(), tets[neg, 1].copy()
    Dm = np.stack([x0[tets[:, k]] - x0[tets[:, 0]] for k in (1, 2, 3)], axis=2)
    vol = np.linalg.det(Dm) / 6.0
    inv = np.linalg.inv(Dm).reshape(-1, 9)
    mu = d.youngs / (1.0 + d.poisson)
    w_rot = mu * vol
    w_vol = w_rot * d.poisson
    N, T = x0.shape[0], tets.shape[0]
    flat = tets.reshape(-1)
    order = np.argsort(flat, kind="stable")            # slots (4t + corner) grouped by vertex, in slot order
    ptr = np.zeros(N + 1, np.int32)
    np.add.at(ptr, flat + 1, 1)
    ptr = np.cumsum(ptr).astype(np.int32)
    return tets, inv, w_rot, w_vol, ptr, order.astype(np.int32)


def test_noalloc_matches_allocating_path_on_two_calls():
    import torch

    d = S.inverse_stiffness(nx=12, ny=4, nz=4)
    d.attach_vertex = np.zeros(0, np.int32)
    d.attach_target = np.zeros((0, 3))
    d.attach_stiffness = np.zeros(0)
    ref = Scene(d)  # the allocating path
    tets, inv, w_rot, w_vol, ptr, slots = raw_arrays(d)
    dev = torch.device("cuda", 0)
    T = lambda a, dt: torch.tensor(np.ascontiguousarray(a), dtype=dt, device=dev)
    t_tets, t_inv = T(tets, torch.int32), T(inv, torch.float64)
    t_wr, t_wv = T(w_rot, torch.float64), T(w_vol, torch.float64)
    t_ptr, t_slot = T(ptr, torch.int32), T(slots, torch.int32)
    out = torch.empty(3 * d.n_vertices, dtype=torch.float64, device=dev)
    rng = np.random.default_rng(11)
    stream = torch.cuda.current_stream(dev)
    for call in range(2):
        x = d.x0.reshape(-1) + 0.02 * rng.standard_normal(3 * d.n_vertices)
        tx = T(x, torch.float64)
        rc = _capi.lib().dfem_eval_corotated_noalloc(
            d.n_vertices, d.n_tets, tx.data_ptr(), t_tets.data_ptr(), t_inv.data_ptr(), t_wr.data_ptr(),
            t_wv.data_ptr(), t_ptr.data_ptr(), t_slot.data_ptr(), out.data_ptr(), stream.cuda_stream)
        _capi.check(rc)
        stream.synchronize()
        got = out.cpu().numpy()
        want = ref.eval_local(x)
        err = np.abs(got - want).max() / np.abs(want).max()
        assert err < TOL, (call, err)


def test_noalloc_reports_an_index_out_of_range_on_the_next_call():
    """A tet vertex index out of range is skipped on the device (no access is
    made through it; the affected outputs are NaN); the next call reports it
    with DFEM_ERR_INVALID, and the call after that runs normally."""
    import torch

    d = S.inverse_stiffness(nx=6, ny=2, nz=2)
    tets, inv, w_rot, w_vol, ptr, slots = raw_arrays(d)
    dev = torch.device("cuda", 0)
    T = lambda a, dt: torch.tensor(np.ascontiguousarray(a), dtype=dt, device=dev)
    bad = tets.copy()
    bad[3, 2] = d.n_vertices  # one past the last vertex
    args = [T(inv, torch.float64), T(w_rot, torch.float64), T(w_vol, torch.float64), T(ptr, torch.int32),
            T(slots, torch.int32)]
    tx = T(d.x0.reshape(-1), torch.float64)
    out = torch.zeros(3 * d.n_vertices, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    lib = _capi.lib()

    def call(t):
        return lib.dfem_eval_corotated_noalloc(d.n_vertices, d.n_tets, tx.data_ptr(), t.data_ptr(),
                                               *[a.data_ptr() for a in args], out.data_ptr(), stream.cuda_stream)

    assert call(T(bad, torch.int32)) == 0
    stream.synchronize()
    got = out.cpu().numpy().reshape(-1, 3)
    assert np.isnan(got[tets[3]]).all() and np.isfinite(np.delete(got, tets[3], axis=0)).all()
    assert call(T(tets, torch.int32)) == 1
    assert b"out of range" in lib.dfem_last_error()
    assert call(T(tets, torch.int32)) == 0
    stream.synchronize()
    assert np.isfinite(out.cpu().numpy()).all()


def test_noalloc_rejects_sizes_beyond_the_static_limit():
    lib = _capi.lib()
    rc = lib.dfem_eval_corotated_noalloc(10, 65536 + 1, None, None, None, None, None, None, None, None, None)
    assert rc == 1
    assert b"DFEM_NOALLOC_MAX_TETS" in lib.dfem_last_error()
