"""F_tet and F_tet_adj: floating-point operations of one corotated tet in the
local step and in the adjoint local step, counted by op_count.cpp (the
engine's templated element math instantiated on a counting scalar) over every
tet of a scene in a deformed state.  Measurement infrastructure: its figures
are the per-tet FLOP counts of the local-step rooflines.

    python oracle/op_count.py [steps]    # inverse-stiffness beam after `steps` oracle steps (default 20)
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path[:] = [p for p in sys.path if os.path.abspath(p or ".") != HERE]  # the package, not this folder
sys.path.insert(0, os.path.dirname(HERE))
LIB = os.path.join(HERE, "liboracle_opcount.so")


def lib():
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(os.path.join(HERE, "op_count.cpp")):
        subprocess.run(["make", "-s", "-C", HERE, "opcount"], check=True)
    L = C.CDLL(LIB)
    L.orc_count_tet_ops.restype = C.c_int
    L.orc_count_tet_ops.argtypes = [C.c_int] + [C.c_void_p] * 5 + [C.POINTER(C.c_longlong)]
    return L


def tet_arrays(d, x):
    """Re-oriented tets (Dfobj.h:474-487), row-major invDm, weights, vertex positions."""
    x0 = d.x0.reshape(-1, 3)
    tets = d.tets.reshape(-1, 4).astype(np.int64).copy()
    Dm = np.stack([x0[tets[:, k]] - x0[tets[:, 0]] for k in (1, 2, 3)], axis=2)
    neg = np.linalg.det(Dm) < 0
    tets[neg, 1], tets[neg, 2] = tets[neg, 2].copy(), tets[neg, 1].copy()
    Dm = np.stack([x0[tets[:, k]] - x0[tets[:, 0]] for k in (1, 2, 3)], axis=2)
    vol = np.linalg.det(Dm) / 6.0
    inv = np.linalg.inv(Dm).reshape(-1, 9)
    E, nu = d.youngs, d.poisson
    wr = E / (1.0 + nu) * vol
    w = np.stack([E, nu, vol, wr, nu * wr], axis=1)
    xs = x.reshape(-1, 3)[tets].reshape(-1, 12)
    return inv, xs, w


def count(d, x, seed=0):
    inv, xs, w = tet_arrays(d, x)
    ys = np.random.default_rng(seed).standard_normal(xs.shape)
    L = lib()
    T = inv.shape[0]
    per = np.zeros((T, 10), np.int64)
    out = (C.c_longlong * 10)()
    for t in range(T):
        a = [np.ascontiguousarray(v[t:t + 1]) for v in (inv, xs, ys, xs, w)]
        L.orc_count_tet_ops(1, *[v.ctypes.data for v in a], out)
        per[t] = list(out)
    return per


def main():
    from diff_fem_b200 import scene as S
    from oracle import oracle as O
    steps = int(sys.argv[1]) if len(sys.argv) > 1 else 20
    d = S.inverse_stiffness()
    x = d.x0.reshape(-1).copy()
    if steps:
        x = O.OracleScene(d).forward(x, np.zeros_like(x), n_steps=steps)["x"]
    per = count(d, x)
    flops = lambda c: c[:, 0] + c[:, 1] + c[:, 2] + c[:, 3]
    for name, c in (("F_tet (local step)", per[:, :5]), ("F_tet_adj (adjoint local step)", per[:, 5:])):
        f = flops(c)
        print(f"{name}: flops per tet mean {f.mean():.1f}, min {f.min()}, max {f.max()}  "
              f"[add {c[:, 0].mean():.1f}, mul {c[:, 1].mean():.1f}, div {c[:, 2].mean():.1f}, "
              f"sqrt/rsqrt {c[:, 3].mean():.1f}, compares {c[:, 4].mean():.1f}]")
    print(f"scene: inverse-stiffness beam, {d.n_tets} tets, state after {steps} oracle steps from rest")


if __name__ == "__main__":
    main()
