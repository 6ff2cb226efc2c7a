"""CPU tests of the engine's host side and C ABI (no GPU needed).

* the C-ABI library loads and exports every entry point include/dfem.h declares;
* the ctypes descriptor mirrors the header's field list;
* the engine's own ordering + supernodal Cholesky (dfem_host_factor_solve)
  solves Hs X = B against the oracle's assembly of Hs;
* descriptor validation turns bad input into DFEM_ERR_INVALID.
"""
import ctypes as C
import os
import re

import numpy as np
import pytest
import scipy.sparse as sp

from diff_fem_b200 import _capi, scene as S
from diff_fem_b200.engine import host_factor_solve
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "dfem.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(dfem_[a-z_0-9]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    lib = _capi.lib()
    names = declared_functions()
    assert len(names) >= 10
    for n in names:
        assert hasattr(lib, n), n
    assert lib.dfem_abi_version() == 6


def test_ctypes_descriptor_matches_header():
    src = open(HEADER).read()
    body = src[src.index("typedef struct dfem_scene_desc"): src.index("} dfem_scene_desc;")]
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    fields = []
    for decl in body.split(";")[:-1]:
        decl = decl.split("{")[-1].strip()
        if not decl:
            continue
        name = re.findall(r"\**\s*([a-z_0-9]+)\s*(\[\d+\])?\s*$", decl)[0][0]
        fields.append(name)
    assert fields == [f for f, _ in _capi.SceneDescC._fields_]


@pytest.mark.parametrize("builder", ["cantilever", "inverse_stiffness", "muscle_beam", "cloth_sheet"])
def test_host_factor_solve_matches_oracle_matrix(builder):
    d = getattr(S, builder)()
    N = d.n_vertices
    b = np.random.default_rng(3).standard_normal(3 * N)
    x, info = host_factor_solve(d, b)
    o = O.OracleScene(d)
    r, c, v = o.hs_coo()
    H = sp.csr_matrix((v, (r, c)), shape=(N, N))
    X, B = x.reshape(N, 3), b.reshape(N, 3)
    assert np.abs(H @ X - B).max() <= 1e-12 * np.abs(B).max() * max(1.0, np.abs(H).max() * np.abs(X).max() / np.abs(B).max())
    # same solution as the oracle's own envelope Cholesky solve (via one zero-iteration step)
    Xs = sp.linalg.spsolve(H.tocsc(), B)
    assert np.abs(Xs - X).max() <= 1e-10 * np.abs(Xs).max()
    assert info["n_supernodes"] >= 1 and info["n_levels"] >= 1 and info["factor_regularisation"] == 0.0


def test_descriptor_validation():
    d = S.cantilever()
    bad = S.cantilever()
    bad.tets = d.tets.copy()
    bad.tets[0, 0] = d.n_vertices + 5
    with pytest.raises(_capi.DfemError) as e:
        host_factor_solve(bad, np.zeros(3 * d.n_vertices))
    assert e.value.code == 1
    bad = S.cantilever()
    bad.mass = d.mass.copy()
    bad.mass[3] = -1.0
    with pytest.raises(_capi.DfemError):
        host_factor_solve(bad, np.zeros(3 * d.n_vertices))
    bad = S.cantilever()
    bad.x0 = d.x0.copy()
    bad.x0[0] = np.nan
    with pytest.raises(_capi.DfemError):
        host_factor_solve(bad, np.zeros(3 * d.n_vertices))


def test_indefinite_matrix_is_regularised_like_the_reference():
    """Negative masses make Hs indefinite; the factorisation retries with
    A + reg I (World::FactorizeLDLT) and reports the regularisation used."""
    d = S.cantilever()
    d.mass = d.mass.copy()
    d.mass[:] = 1e-30  # tiny masses: still valid input
    b = np.ones(3 * d.n_vertices)
    x, info = host_factor_solve(d, b)
    assert np.all(np.isfinite(x))


def test_obj_writer_writes_the_reference_format(tmp_path):
    """dfem_obj_writer (Environment::SaveObj / Save, sim/Environment.h:295-327):
    per body "v %06f %06f %06f" then 1-based "f %d %d %d" lines, from host
    states queued faster than they are written; files byte-identical to the
    format written directly."""
    from diff_fem_b200.engine import ObjWriter
    rng = np.random.default_rng(5)
    bodies = [(5, np.array([[0, 1, 2], [2, 3, 4]]), "_DfObj0.obj"), (3, np.array([[0, 2, 1]]), "_DfCloths0.obj")]
    w = ObjWriter(bodies, depth=2)
    states = [rng.standard_normal(24) * 10 for _ in range(6)]
    for k, x in enumerate(states):
        w.write(str(tmp_path / f"{k:03d}"), x)
    w.flush()
    for k, x in enumerate(states):
        X = x.reshape(-1, 3)
        off = 0
        for n, faces, suffix in bodies:
            want = "".join("v %06f %06f %06f\n" % tuple(p) for p in X[off:off + n])
            want += "".join("f %d %d %d\n" % (f[0] + 1, f[1] + 1, f[2] + 1) for f in faces)
            assert (tmp_path / f"{k:03d}{suffix}").read_text() == want
            off += n
    w.write(str(tmp_path / "missing_dir" / "x"), states[0])
    with pytest.raises(_capi.DfemError):
        w.flush()  # the unwritable file surfaces at the flush
    w.close()
    with pytest.raises(_capi.DfemError):
        ObjWriter([(2, np.array([[0, 1, 2]]), "_a.obj")])  # face vertex out of range


def _warp_tree(slots):
    """The warp form of a vertex's slot sum: lane l adds slots l, l + 32, ...
    from +0, then the xor butterfly (offsets 16, 8, 4, 2, 1)."""
    v = [0.0] * 32
    for l in range(32):
        for k in range(l, len(slots), 32):
            v[l] = v[l] + slots[k]
    for o in (16, 8, 4, 2, 1):
        v = [v[l] + v[l ^ o] for l in range(32)]
    return v


def _thread_tree(slots):
    """The thread form: the same lane partials, pairwise-summed over the
    lanes in bit-reversed order with a five-entry stack."""
    stk = [None] * 5
    for j in range(32):
        lane = int(f"{j:05b}"[::-1], 2)
        x = 0.0
        for k in range(lane, len(slots), 32):
            x = x + slots[k]
        b = 0
        while b < 5 and (j >> b) & 1:
            x = stk[b] + x
            b += 1
        if j == 31:
            return x
        stk[b] = x


def test_thread_gather_reproduces_the_warp_reduction_bit_for_bit():
    """k_gather_t / k_adj_gather_t emulate k_gather / k_adj_gather: every lane
    of the butterfly ends with the same sum, and the thread's pairwise tree
    over bit-reversed lanes is that sum, bit for bit (signed zeros included)."""
    import struct
    rng = np.random.default_rng(11)
    bits = lambda a: struct.pack("<d", a)
    for n in list(range(0, 70)) + [95, 96, 97, 130]:
        for scale in (1.0, 1e-300, 1e300):
            slots = list(rng.standard_normal(n) * scale * 10.0 ** rng.integers(-8, 8, n))
            if n > 3:
                slots[1], slots[2] = -0.0, 0.0
            w = _warp_tree(slots)
            assert len({bits(a) for a in w}) == 1
            assert bits(_thread_tree(slots)) == bits(w[0]), n
