"""ctypes binding of the CPU FP64 oracle (liboracle_pd.so).

TEST INFRASTRUCTURE ONLY: the checker the CUDA engine is compared against.
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs may
import this module; the product package never does.

PARITY UNPINNED against the reference binary (diff_fem cannot be built or
imported here: Eigen, CppAD, CGAL and Boost are absent).  See pd_oracle.cpp.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle_pd.so")

_lib = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        vp, pd, pi = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int)
        L.orc_create.restype = vp
        L.orc_create.argtypes = [C.c_void_p]
        L.orc_destroy.argtypes = [vp]
        L.orc_regularisation.restype = C.c_double
        L.orc_regularisation.argtypes = [vp]
        L.orc_set_materials.argtypes = [vp, pd, pd]
        L.orc_forward.argtypes = [vp, pd, pd, pd, C.c_int, pd, pd, pd, pi, C.c_int]
        L.orc_backward.argtypes = [vp, pd, pd, pd, pd, pd, pd, pd]
        L.orc_lumped_masses.argtypes = [C.c_int, pd, C.c_int, pi, C.c_double, C.c_int, pd]
        L.orc_eval_local.argtypes = [vp, pd, pd, pd]
        L.orc_contact_passes.argtypes = [vp, pi, C.c_int]
        L.orc_set_detection_replay.argtypes = [vp, C.c_int]
        L.orc_self_group.argtypes = [pd, pd, pd, C.c_int, C.c_double, pd, pi]
        L.orc_vf_impact.argtypes = [pd, pd, pd, pd, pd, C.c_double, pd]
        L.orc_corot_project.argtypes = [pd, pd, pd]
        L.orc_corot_vjp.argtypes = [pd, pd, pd, pd]
        L.orc_svd3.argtypes = [pd, pd, pd, pd]
        L.orc_hs_coo.restype = C.c_int64
        L.orc_hs_coo.argtypes = [vp, pi, pi, pd, C.c_int64]
        L.orc_full_L_triplets.restype = C.c_int64
        L.orc_full_L_triplets.argtypes = [vp, pi, pi, pd, C.c_int64]
        L.orc_joint_state_size.argtypes = [vp]
        L.orc_set_joint_state.argtypes = [vp, pd, pd]
        L.orc_get_joint_state.argtypes = [vp, pd, pd]
        _lib = L
    return _lib


def _pd(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_double))


def _pi(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_int))


class OracleScene:
    """FP64 CPU restatement of one diff_fem world (no contact phase)."""

    def __init__(self, desc):
        self.desc = desc
        cdesc, self._keep = desc.to_c()
        self.h = lib().orc_create(C.byref(cdesc))
        if not self.h:
            raise RuntimeError("oracle: scene creation / factorisation failed")
        self.N = desc.n_vertices
        self.T = desc.n_tets
        self.nseg = int(desc.n_segments)
        self._steps = 0

    def __del__(self):
        if getattr(self, "h", None) and lib is not None:  # module globals may be gone at interpreter exit
            try:
                lib().orc_destroy(self.h)
            except Exception:
                pass
            self.h = None

    @property
    def regularisation(self) -> float:
        return lib().orc_regularisation(self.h)

    def set_materials(self, E, nu):
        E = np.ascontiguousarray(E, np.float64)
        nu = np.ascontiguousarray(nu, np.float64)
        rc = lib().orc_set_materials(self.h, _pd(E), _pd(nu))
        if rc:
            raise RuntimeError(f"oracle: set_materials failed ({rc})")

    def forward(self, x, v, n_steps=1, act=None, traj=False, threads=1):
        n3 = 3 * self.N
        x = np.ascontiguousarray(x, np.float64).reshape(-1)
        v = np.ascontiguousarray(v, np.float64).reshape(-1)
        xo, vo = np.zeros(n3), np.zeros(n3)
        tr = np.zeros((n_steps, n3)) if traj else None
        it = np.zeros(n_steps, np.int32)
        a = None if act is None else np.ascontiguousarray(act, np.float64).reshape(-1)
        rc = lib().orc_forward(self.h, _pd(x), _pd(v), _pd(a), int(n_steps), _pd(xo), _pd(vo), _pd(tr), _pi(it), int(threads))
        if rc:
            raise RuntimeError(f"oracle: forward failed ({rc})")
        self._steps = n_steps
        out = {"x": xo, "v": vo, "iters": it}
        if traj:
            out["traj"] = tr
        return out

    def backward(self, gx, gv):
        n3 = 3 * self.N
        gx = np.ascontiguousarray(gx, np.float64).reshape(-1)
        gv = np.ascontiguousarray(gv, np.float64).reshape(-1)
        ox, ov = np.zeros(n3), np.zeros(n3)
        gE, gnu = np.zeros(max(1, self.T)), np.zeros(max(1, self.T))
        ga = np.zeros(max(1, self._steps * self.nseg))
        rc = lib().orc_backward(self.h, _pd(gx), _pd(gv), _pd(ox), _pd(ov), _pd(gE), _pd(gnu), _pd(ga))
        if rc:
            raise RuntimeError(f"oracle: backward failed ({rc})")
        return {"x": ox, "v": ov, "E": gE[: self.T], "nu": gnu[: self.T],
                "act": ga[: self._steps * self.nseg].reshape(self._steps, self.nseg)}

    def joint_state(self):
        """(jq, jqd): World::mJointQ / mJointQd of the skeleton (empty without links)."""
        n = lib().orc_joint_state_size(self.h)
        jq, jqd = np.zeros(max(1, n)), np.zeros(max(1, n))
        if n:
            lib().orc_get_joint_state(self.h, _pd(jq), _pd(jqd))
        return jq[:n], jqd[:n]

    def set_joint_state(self, jq, jqd):
        n = lib().orc_joint_state_size(self.h)
        jq = np.ascontiguousarray(jq, np.float64).reshape(-1)
        jqd = np.ascontiguousarray(jqd, np.float64).reshape(-1)
        if jq.size != n or jqd.size != n:
            raise ValueError(f"joint state needs {n} values each")
        if n:
            lib().orc_set_joint_state(self.h, _pd(jq), _pd(jqd))

    def eval_local(self, x, act=None):
        """J d(x) of all constraints (3N)."""
        x = np.ascontiguousarray(x, np.float64).reshape(-1)
        a = None if act is None else np.ascontiguousarray(act, np.float64).reshape(-1)
        out = np.zeros(3 * self.N)
        lib().orc_eval_local(self.h, _pd(x), _pd(a), _pd(out))
        return out

    def detection_replay(self, mode: int):
        """0: detect; 1: record each step's contact passes (impact normals,
        self groups) on the next forward; 2: replay the recorded passes."""
        lib().orc_set_detection_replay(self.h, int(mode))

    def contact_passes(self):
        out = np.zeros(max(1, self._steps), np.int32)
        lib().orc_contact_passes(self.h, _pi(out), self._steps)
        return out[: self._steps]

    def hs_coo(self):
        cap = lib().orc_hs_coo(self.h, None, None, None, 0)
        r, c, v = np.zeros(cap, np.int32), np.zeros(cap, np.int32), np.zeros(cap)
        lib().orc_hs_coo(self.h, _pi(r), _pi(c), _pd(v), cap)
        return r, c, v

    def full_L_triplets(self):
        cap = lib().orc_full_L_triplets(self.h, None, None, None, 0)
        r, c, v = np.zeros(cap, np.int32), np.zeros(cap, np.int32), np.zeros(cap)
        lib().orc_full_L_triplets(self.h, _pi(r), _pi(c), _pd(v), cap)
        return r, c, v


def corot_project(F):
    F = np.asfortranarray(F, np.float64)
    md = np.zeros((3, 3), order="F")
    mdv = np.zeros((3, 3), order="F")
    lib().orc_corot_project(_pd(F), _pd(md), _pd(mdv))
    return np.array(md), np.array(mdv)


def corot_vjp(F, gmd, gmdv):
    F = np.asfortranarray(F, np.float64)
    a = np.asfortranarray(gmd, np.float64)
    b = np.asfortranarray(gmdv, np.float64)
    out = np.zeros((3, 3), order="F")
    lib().orc_corot_vjp(_pd(F), _pd(a), _pd(b), _pd(out))
    return np.array(out)


def svd3(F):
    F = np.asfortranarray(F, np.float64)
    U = np.zeros((3, 3), order="F")
    V = np.zeros((3, 3), order="F")
    s = np.zeros(3)
    lib().orc_svd3(_pd(F), _pd(U), _pd(s), _pd(V))
    return np.array(U), s, np.array(V)


def vf_impact(p0, p1, q0, q1, q2, mult=1.0):
    """One vertex-face CCD test; returns (hit, normal)."""
    a = [np.ascontiguousarray(v, np.float64) for v in (p0, p1, q0, q1, q2)]
    n = np.zeros(3)
    hit = lib().orc_vf_impact(*[_pd(v) for v in a], float(mult), _pd(n))
    return bool(hit), n


def lumped_masses(x0, tets, total_mass, is_mass_same=True):
    x0 = np.ascontiguousarray(x0, np.float64).reshape(-1)
    tets = np.ascontiguousarray(tets, np.int32).reshape(-1)
    n = x0.size // 3
    m = np.zeros(n)
    lib().orc_lumped_masses(n, _pd(x0), tets.size // 4, _pi(tets), float(total_mass), int(is_mass_same), _pd(m))
    return m


def self_group(normal, P, m, mu):
    """One soft-contact face group's exchange: P = (3 + k, 3) forces of the
    face's vertices then of the group's k vertices, m their masses.  Returns
    (self forces (3 + k, 3), membership of the k group vertices)."""
    P = np.ascontiguousarray(P, np.float64).reshape(-1, 3)
    m = np.ascontiguousarray(m, np.float64)
    k = P.shape[0] - 3
    out = np.zeros_like(P)
    inc = np.zeros(max(1, k), np.int32)
    lib().orc_self_group(_pd(np.ascontiguousarray(normal, np.float64)), _pd(P), _pd(m), k, float(mu), _pd(out), _pi(inc))
    return out, inc[:k].astype(bool)
