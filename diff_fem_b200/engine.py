"""Python handle over one engine scene (C-ABI calls through ctypes).

Buffers may be numpy arrays (host, FP64) or torch tensors (host or CUDA, FP64,
contiguous); CUDA tensors are passed to the engine as device pointers, so a
step reads and writes HBM directly with no host round trip.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import _capi
from ._capi import DFEM_MEM_DEVICE, DFEM_MEM_HOST, check, lib

try:  # torch is optional for the host-array path
    import torch
except Exception:  # pragma: no cover
    torch = None


def _is_cuda_tensor(a) -> bool:
    return torch is not None and isinstance(a, torch.Tensor) and a.is_cuda


def _sync_torch(*arrays):
    """Make pending work of torch's current stream visible to the engine's stream."""
    for a in arrays:
        if _is_cuda_tensor(a):
            torch.cuda.current_stream(a.device).synchronize()
            return


def _ptr(a):
    """(pointer, mem kind, keepalive) of a numpy array or torch tensor (FP64)."""
    if a is None:
        return None, None, None
    if torch is not None and isinstance(a, torch.Tensor):
        if a.dtype != torch.float64 or not a.is_contiguous():
            raise TypeError("engine buffers must be contiguous float64 tensors")
        return a.data_ptr(), (DFEM_MEM_DEVICE if a.is_cuda else DFEM_MEM_HOST), a
    arr = np.ascontiguousarray(a, dtype=np.float64)
    return arr.ctypes.data, DFEM_MEM_HOST, arr


class Scene:
    """One simulated world on one GPU (an opaque ``dfem_scene``), or a batch
    of independent worlds stepped together (``Scene.batch``)."""

    def __init__(self, desc, device: int = 0):
        self.desc = desc
        cdesc, keep = desc.to_c()
        h = C.c_void_p()
        check(lib().dfem_scene_create(C.byref(cdesc), int(device), C.byref(h)))
        self._init_handle(h, device)

    @classmethod
    def batch(cls, descs, device: int = 0) -> "Scene":
        """Independent scenes as one handle: x, v, materials, activations and
        gradients are the concatenation of the scenes' arrays (``offsets``
        gives each part's first vertex, tet and segment); every part keeps its
        own convergence test and iteration count."""
        descs = list(descs)
        arr = (_capi.SceneDescC * len(descs))()
        keep = []
        for i, d in enumerate(descs):
            c, k = d.to_c()
            arr[i] = c
            keep.append((c, k))
        h = C.c_void_p()
        check(lib().dfem_scene_create_batch(arr, len(descs), int(device), C.byref(h)))
        self = cls.__new__(cls)
        self.desc = descs
        self._init_handle(h, device)
        return self

    def _init_handle(self, h, device):
        self._h = h
        self.device = device
        n = C.c_int32()
        check(lib().dfem_batch_layout(h, C.byref(n), None, None, None))
        self.nparts = int(n.value)
        vo, to, so = (np.zeros(self.nparts + 1, np.int32) for _ in range(3))
        P = lambda a: a.ctypes.data_as(C.POINTER(C.c_int32))
        check(lib().dfem_batch_layout(h, C.byref(n), P(vo), P(to), P(so)))
        self.offsets = {"vertices": vo, "tets": to, "segments": so}
        self.N = int(vo[-1])
        self.T = int(to[-1])
        self.nseg = int(so[-1])
        self._last_steps = 0

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().dfem_scene_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def info(self) -> dict:
        inf = _capi.SceneInfoC()
        check(lib().dfem_scene_get_info(self._h, C.byref(inf)))
        return {name: getattr(inf, name) for name, _ in inf._fields_}

    def set_materials(self, youngs, poisson):
        pe, me, ke = _ptr(youngs)
        pn, mn, kn = _ptr(poisson)
        if me != mn:
            raise ValueError("youngs and poisson must live in the same memory")
        _sync_torch(youngs, poisson)
        check(lib().dfem_set_materials(self._h, pe, pn, me))

    def set_activations(self, act):
        p, m, k = _ptr(act)
        check(lib().dfem_set_activations(self._h, p, m))

    @property
    def n_joint_state(self) -> int:
        """Length of the skeleton's joint state (12 + links - 1), 0 without links."""
        d = self.desc if not isinstance(self.desc, list) else None
        nl = int(np.asarray(d.link_parent).size) if d is not None else 0
        return 12 + nl - 1 if nl else 0

    def joint_state(self):
        """(jq, jqd): World::mJointQ / mJointQd of the skeleton after the last
        forward call (the root's T, row-major R then d, and the other links'
        magnitudes; jqd the previous step's)."""
        n = self.n_joint_state
        jq, jqd = np.zeros(n), np.zeros(n)
        if n:
            P = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
            check(lib().dfem_get_joint_state(self._h, P(jq), P(jqd)))
        return jq, jqd

    def set_joint_state(self, jq, jqd):
        n = self.n_joint_state
        jq = np.ascontiguousarray(jq, np.float64).reshape(-1)
        jqd = np.ascontiguousarray(jqd, np.float64).reshape(-1)
        if jq.size != n or jqd.size != n:
            raise ValueError(f"joint state needs {n} values each")
        if n:
            P = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
            check(lib().dfem_set_joint_state(self._h, P(jq), P(jqd)))

    def forward(self, x, v, n_steps: int = 1, act=None, traj: bool = False):
        """Run n_steps steps from (x, v).  Returns (x_out, v_out[, traj]) in the
        input's memory kind (numpy for host input, CUDA tensors for device input)."""
        dev = _is_cuda_tensor(x)
        n3 = 3 * self.N
        if dev:
            xo = torch.empty(n3, dtype=torch.float64, device=x.device)
            vo = torch.empty_like(xo)
            tr = torch.empty((n_steps, n3), dtype=torch.float64, device=x.device) if traj else None
        else:
            xo, vo = np.empty(n3), np.empty(n3)
            tr = np.empty((n_steps, n3)) if traj else None
        px, mx, kx = _ptr(x)
        pv, mv, kv = _ptr(v)
        pa, ma, ka = _ptr(act)
        pxo, _, _ = _ptr(xo)
        pvo, _, _ = _ptr(vo)
        ptr_, _, _ = _ptr(tr)
        if mx != mv or (ma is not None and ma != mx):
            raise ValueError("x, v and act must live in the same memory")
        _sync_torch(x, v, act)
        check(lib().dfem_step_forward(self._h, px, pv, pa, int(n_steps), pxo, pvo, ptr_, mx))
        self._last_steps = n_steps
        return (xo, vo, tr) if traj else (xo, vo)

    def backward(self, gx, gv, gjq=None, gjqd=None):
        """VJP of the last forward call.  Returns dict with x, v, E, nu, act;
        with a skeleton also jq, jqd (the gradient w.r.t. the joint state the
        forward started from; gjq / gjqd: cotangents of its end state, zero
        when omitted)."""
        nq = self.n_joint_state
        if nq and (gjq is not None or gjqd is not None):
            a = np.zeros(nq) if gjq is None else np.ascontiguousarray(gjq, np.float64).reshape(-1)
            b = np.zeros(nq) if gjqd is None else np.ascontiguousarray(gjqd, np.float64).reshape(-1)
            if a.size != nq or b.size != nq:
                raise ValueError(f"joint state cotangents need {nq} values each")
            P = lambda t: t.ctypes.data_as(C.POINTER(C.c_double))
            check(lib().dfem_set_joint_state_grad(self._h, P(a), P(b)))
        dev = _is_cuda_tensor(gx)
        n3 = 3 * self.N
        if dev:
            mk = lambda *s: torch.empty(*s, dtype=torch.float64, device=gx.device)
        else:
            mk = lambda *s: np.empty(s if len(s) > 1 else s[0])
        ox, ov = mk(n3), mk(n3)
        gE, gnu = mk(max(1, self.T)), mk(max(1, self.T))
        ga = mk(max(1, self._last_steps * self.nseg))
        p = [_ptr(a)[0] for a in (gx, gv, ox, ov, gE, gnu, ga)]
        mem = _ptr(gx)[1]
        _sync_torch(gx, gv)
        check(lib().dfem_step_backward(self._h, p[0], p[1], p[2], p[3], p[4], p[5], p[6] if self.nseg else None, mem))
        act = ga[: self._last_steps * self.nseg]
        act = act.reshape(self._last_steps, self.nseg)
        out = {"x": ox, "v": ov, "E": gE[: self.T], "nu": gnu[: self.T], "act": act}
        if nq:
            ja, jb = np.zeros(nq), np.zeros(nq)
            P = lambda t: t.ctypes.data_as(C.POINTER(C.c_double))
            check(lib().dfem_get_joint_state_grad(self._h, P(ja), P(jb)))
            out["jq"], out["jqd"] = ja, jb
        return out

    def eval_local(self, x):
        """J d(x): the local step's contribution to the global rhs at positions x."""
        dev = _is_cuda_tensor(x)
        out = torch.empty(3 * self.N, dtype=torch.float64, device=x.device) if dev else np.empty(3 * self.N)
        px, mx, kx = _ptr(x)
        po, _, _ = _ptr(out)
        _sync_torch(x)
        check(lib().dfem_eval_local(self._h, px, po, mx))
        return out

    def iterations(self, n: Optional[int] = None) -> np.ndarray:
        """PD iterations per step of the last forward call: shape (n,) for a
        single scene, (n, parts) for a batch."""
        n = self._last_steps if n is None else n
        out = np.zeros(n * self.nparts, np.int32)
        check(lib().dfem_get_iterations(self._h, out.ctypes.data_as(C.POINTER(C.c_int32)), int(n)))
        return out if self.nparts == 1 else out.reshape(n, self.nparts)

    def contact_passes(self, n: Optional[int] = None) -> np.ndarray:
        n = self._last_steps if n is None else n
        out = np.zeros(n, np.int32)
        check(lib().dfem_get_contact_passes(self._h, out.ctypes.data_as(C.POINTER(C.c_int32)), int(n)))
        return out

    def solve_mode(self, request: Optional[str] = None) -> dict:
        """Form of the global solve: request None (query), "auto" (re-tune),
        "levels", "persistent", "split" (level kernels below the autotuned
        cut level, one persistent launch above), "cluster" (one thread-block
        cluster walks the levels), "resident" (the factor held in one
        cluster's shared memory) or "dense" (one product with Hs^-1, rebuilt
        from the factor after every refactorisation; single scenes up to 4,096
        vertices).  Returns the form in use and the autotune's ms per solve of
        each form."""
        req = {None: -1, "auto": 0, "levels": 1, "persistent": 2, "split": 3, "cluster": 4, "resident": 5,
               "dense": 6}[request]
        chosen = C.c_int32()
        ms = (C.c_double * 2)()
        check(lib().dfem_solve_mode(self._h, req, C.byref(chosen), ms))
        cut, nl, mss = C.c_int32(), C.c_int32(), C.c_double()
        check(lib().dfem_solve_split(self._h, C.byref(cut), C.byref(nl), C.byref(mss)))
        on, thr, one = C.c_int32(), C.c_double(), (C.c_double * 2)()
        check(lib().dfem_solve_select(self._h, C.byref(on), C.byref(thr), one))
        t6 = (C.c_double * 7)()
        check(lib().dfem_solve_times(self._h, t6, 7))
        return {"mode": {1: "levels", 2: "persistent", 3: "split", 4: "cluster", 5: "resident",
                         6: "dense"}[chosen.value],
                "ms_levels": ms[0], "ms_cluster": t6[3], "ms_resident": t6[4], "ms_dense": t6[5], "ms_dense_build": t6[6],
                "ms_persistent": ms[1], "ms_split": mss.value, "split_level": cut.value, "levels": nl.value,
                "tail_persistent_below": thr.value if on.value else None,
                "ms_largest_part_only": [one[0], one[1]]}

    def profile_levels(self, reps: int = 10) -> dict:
        """ms per launch of every forward / backward launch of the level-kernel
        solve (a level, split into its small and large supernodes), with the
        supernodes, level and CTA sizes of each launch."""
        n = C.c_int32()
        check(lib().dfem_profile_levels(self._h, int(reps), 0, C.byref(n), None, None, None, None, None))
        G = int(n.value)
        f, b = (C.c_double * G)(), (C.c_double * G)()
        cnt, lvl, thr = (C.c_int32 * G)(), (C.c_int32 * G)(), (C.c_int32 * (2 * G))()
        check(lib().dfem_profile_levels(self._h, int(reps), G, C.byref(n), f, b, cnt, lvl, thr))
        return {"fwd_ms": list(f), "bwd_ms": list(b), "supernodes": list(cnt), "level": list(lvl),
                "threads_fwd": list(thr)[0::2], "threads_bwd": list(thr)[1::2]}

    LIMITS = {"contact_passes": 0, "impacts_per_vertex": 1, "soft_impacts_per_vertex": 2, "group_members": 3,
              "solve_wait_polls": 4, "broad_phase_cells": 5}

    def set_limit(self, which: str, value: int = -1):
        """Lower one of the engine's caps for this scene (value < 0: the
        built-in cap again); a call that reaches it raises DfemError with
        DFEM_ERR_CAP.  See dfem_set_limit."""
        check(lib().dfem_set_limit(self._h, self.LIMITS[which], int(value)))

    OPTIONS = {"fused_contact": 0, "split_factor": 1, "gather": 2}

    def set_option(self, which: str, value: int):
        """An execution option (results are identical either way); see dfem_set_option."""
        check(lib().dfem_set_option(self._h, self.OPTIONS[which], int(value)))

    def set_adjoint_budget(self, nbytes: int):
        """Device memory for storing every step's iterates (the adjoint then replays no step)."""
        check(lib().dfem_set_adjoint_budget(self._h, int(nbytes)))

    def launch_count(self) -> int:
        n = C.c_int64()
        check(lib().dfem_get_launch_count(self._h, C.byref(n)))
        return int(n.value)

    def profile_phases(self, reps: int = 20) -> dict:
        ms = (C.c_double * 4)()
        check(lib().dfem_profile_phases(self._h, int(reps), ms))
        return {"local": ms[0], "gather": ms[1], "solve": ms[2], "adj_local": ms[3]}

    def synchronize(self):
        check(lib().dfem_synchronize(self._h))


def host_factor_solve(desc, b) -> tuple:
    """Host-only diagnostic: solve Hs X = B with the engine's own ordering and
    supernodal factor (no GPU).  Returns (X (3N,), info dict)."""
    cdesc, keep = desc.to_c()
    b = np.ascontiguousarray(b, np.float64).reshape(-1)
    x = np.empty_like(b)
    inf = _capi.SceneInfoC()
    check(lib().dfem_host_factor_solve(C.byref(cdesc), b.ctypes.data, x.ctypes.data, C.byref(inf)))
    return x, {name: getattr(inf, name) for name, _ in inf._fields_}


class ObjWriter:
    """Asynchronous per-step OBJ output (dfem_obj_writer_*): Environment::SaveObj
    / Save (sim/Environment.h:295-327) as a queue of staging slots drained by a
    host thread.  bodies: list of (vertex_count, faces (F, 3) body-local ids,
    file-name suffix); states are 3N in the bodies' order, numpy (host) or
    CUDA tensors (copied on the scene's stream)."""

    def __init__(self, bodies, depth: int = 4):
        nv = [int(b[0]) for b in bodies]
        fc = [np.asarray(b[1], np.int32).reshape(-1, 3) for b in bodies]
        self._voff = np.cumsum([0] + nv).astype(np.int32)
        self._foff = np.cumsum([0] + [f.shape[0] for f in fc]).astype(np.int32)
        self._faces = np.ascontiguousarray(np.concatenate(fc) if fc else np.zeros((0, 3), np.int32), np.int32)
        self._suffix = (C.c_char_p * len(bodies))(*[str(b[2]).encode() for b in bodies])
        P = lambda a: a.ctypes.data_as(C.POINTER(C.c_int32))
        h = C.c_void_p()
        check(lib().dfem_obj_writer_create(len(bodies), P(self._voff), P(self._foff), P(self._faces),
                                           self._suffix, int(depth), C.byref(h)))
        self._h = h
        self._keep = []

    def write(self, prefix: str, x, scene: Optional["Scene"] = None):
        p, m, keep = _ptr(x)
        if m == DFEM_MEM_DEVICE:
            if scene is None:
                raise ValueError("a device state needs the scene whose stream produced it")
            _sync_torch(x)
        check(lib().dfem_obj_writer_enqueue(self._h, scene.handle if scene is not None else None,
                                            str(prefix).encode(), p, m))

    def flush(self):
        check(lib().dfem_obj_writer_flush(self._h))

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().dfem_obj_writer_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
