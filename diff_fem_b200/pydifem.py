"""The ``pydifem`` module surface of diff_fem, served by the CUDA engine.

Same functions, argument order and meaning as the reference's pybind11 module
(python/pydifem.cc:329-389):

    init_env(total_step, config_path) -> Environment
    forward_act(q, qd, jq, jqd, tau, env, is_act) -> [q, qd, jq, jqd]
    backward_act(q, qd, jq, jqd, tau, dldq, dldqd, dldjq, dldjqd, env, is_act)
        -> [dq, dqd, djq, djqd, dtau]
    forward_all(q, qd, tau, env) -> [q, qd]          (tau[0] = E, tau[1] = nu for every tet)
    backward_all(q, qd, tau, dldq, dldqd, env) -> [dq, dqd, dtau]
    vector2double(v) -> list, double2vector(list) -> vector

Differences: values are FP64 numpy arrays (the reference returns float lists
that api_diff.py truncates to float32); gradients come from the engine's
adjoint instead of a CppAD tape, through an articulated skeleton's links too
(djq, djqd from dldjq, dldjqd; the joint torques of actuator type 1 in
dtau).  The actuator front-end of type 2 (muscles:
Normalizer::NormToReal, Muscle::SetActivationLevels with the SetKey table,
sim/Normalizer.h:94-112, sim/Muscle.h:224-261, sim/Dfobj.h:628-667) is
evaluated with torch so that dL/dtau follows from the engine's dL/d(activation);
type 3 (pneumatic springs, sim/Dfobj.h:326-330) maps tau to the springs'
activation channels one to one.
"""
from __future__ import annotations

import os
from typing import List, Optional

import numpy as np

from . import loader
from .engine import ObjWriter, Scene

try:
    import torch
except Exception:  # pragma: no cover
    torch = None


def _is_cuda(a) -> bool:
    return torch is not None and isinstance(a, torch.Tensor) and a.is_cuda


def vector2double(v) -> List[float]:
    return [float(a) for a in np.asarray(v, np.float64).reshape(-1)]


def double2vector(v) -> np.ndarray:
    return np.asarray(v, np.float64).reshape(-1).copy()


class World:
    """Mirror of the attributes callers use on FEM::World (pydifem.cc:361-367)."""

    def __init__(self, x0: np.ndarray, h: float):
        self.mX = x0.reshape(-1).copy()
        self.mV = np.zeros_like(self.mX)
        self.mJointQ = np.zeros(0)
        self.mJointQd = np.zeros(0)
        self.mJointTorque = np.zeros(0)
        self._h = h

    def GetTimeStep(self) -> float:
        return self._h


_KEY_ROWS = [(0, 20, (0.025, -0.0625)), (20, 30, (-0.125, 0.03125)), (30, 50, (0.0, -0.125))]


def _muscle_keys(n_muscles: int) -> np.ndarray:
    """Dfobj::SetKey: a 50 x n table of cumulative, clamped increments.  The
    reference writes rows of exactly 16 alternating values; muscles beyond the
    16th reuse the pattern."""
    inc = np.zeros((50, n_muscles))
    for r0, r1, (even, odd) in _KEY_ROWS:
        for j in range(n_muscles):
            inc[r0:r1, j] = even if j % 2 == 0 else odd
    key = np.zeros_like(inc)
    for j in range(n_muscles):
        acc = 0.0
        for i in range(50):
            acc = inc[i, j] if i == 0 else key[i - 1, j] + inc[i, j]
            key[i, j] = min(max(acc, 0.0), 1.0)
    return key


class Dfobj:
    """Mirror of Dfobj (pydifem.cc:369-373): actions, unknowns, activation levels."""

    REAL_LO = np.array([-0.25, 0.0, 0.0, 0.0])
    REAL_HI = np.array([0.25, 1.0, 1.0, 10.0])

    def __init__(self, body: loader.Body):
        self.body = body
        self.mNumUnknown = 3 * body.n
        self.n_muscles = body.n_muscles
        n_act = {1: max(0, body.n_links - 1), 2: 4 * self.n_muscles, 3: body.n_pneumatic}.get(body.actuator_type, 0)
        self.mActions = np.zeros(n_act)
        self.levels = np.zeros((self.n_muscles, 50))
        # PneumaticConstraint::mActivationLevel starts at 1 (pneumaticEasy.h:31)
        self.pneumatic_levels = np.ones(body.n_pneumatic)
        # World::mJointTorque of the non-root links (World.h:372-373: zero at start)
        self.torques = np.zeros(max(0, body.n_links - 1))
        self.keys = _muscle_keys(self.n_muscles) if self.n_muscles else np.zeros((50, 0))

    def GetActivationLevelsAggregate(self) -> np.ndarray:
        return self.levels.reshape(-1).copy()

    def SetActivationLevelsAggregate(self, v) -> None:
        self.levels = np.asarray(v, np.float64).reshape(self.n_muscles, 50).copy()

    def activation_from_actions(self, tau, phase: int, prev):
        """Normalizer::NormToReal + Muscle::SetActivationLevels (torch, differentiable)."""
        lo = torch.tensor(self.REAL_LO, dtype=tau.dtype)
        hi = torch.tensor(self.REAL_HI, dtype=tau.dtype)
        out = []
        for m in range(self.n_muscles):
            a = tau[4 * m: 4 * m + 4]
            real = lo + (hi - lo) * torch.clamp((a + 5.0) / 10.0, 0.0, 1.0)
            key = float(self.keys[phase % 50, m])
            delta, alpha, speed = real[0], real[1], float(real[3].detach())
            beta = 1.0 - alpha
            prev_m = prev[m]
            new = prev_m
            i = 0
            while i < speed:
                first = (key + delta).reshape(1)
                rest = alpha * prev_m[:-1] + beta * prev_m[1:]
                new = torch.cat([first, rest])
                prev_m = new
                i += 1
            out.append(torch.clamp(new, 0.0, 1.0))
        return torch.stack(out) if out else torch.zeros((0, 50), dtype=tau.dtype)


class Environment:
    """Mirror of Environment (pydifem.cc:375-380) backed by one engine scene."""

    def __init__(self, loaded: loader.LoadedScene, device: int = 0):
        self.loaded = loaded
        self.desc = loaded.desc
        self.scene = Scene(self.desc, device=device)
        self.mSoftWorld = World(self.desc.x0, self.desc.time_step)
        self.mDfobjs = [Dfobj(b) for b in loaded.bodies if b.kind == "mesh"]
        self.mPhase = 0
        self.total_step = loaded.total_step
        self._jq0 = self.scene.joint_state()[0]  # World::Initialize: the links' WriteT (World.h:369-370)
        self.mSoftWorld.mJointQ = self._jq0.copy()
        self.mSoftWorld.mJointQd = self._jq0.copy()
        self.mSoftWorld.mJointTorque = np.zeros(max(0, self._jq0.size - 12))
        self._obj = None  # the OBJ writer, made on the first SaveObj
        self._E = np.asarray(self.desc.youngs, np.float64).copy()
        self._nu = np.asarray(self.desc.poisson, np.float64).copy()

    # activation channels of the engine: every body's muscle segments at its
    # seg_offset, its pneumatic springs at its pneumatic_offset
    def segment_activations(self) -> np.ndarray:
        out = np.zeros(self.desc.n_segments)
        for o in self.mDfobjs:
            if o.n_muscles:  # the flattened level table over the body's segments (truncated or zero-padded)
                lv = o.levels.reshape(-1)[: o.body.n_segments]
                out[o.body.seg_offset:o.body.seg_offset + lv.size] = lv
            if o.body.n_pneumatic:
                out[o.body.pneumatic_offset:o.body.pneumatic_offset + o.body.n_pneumatic] = o.pneumatic_levels
            if o.torques.size:
                out[o.body.torque_offset:o.body.torque_offset + o.torques.size] = o.torques
        return out

    def SetActions(self, tau) -> None:
        """Dfobj::SetActions (sim/Dfobj.h:315-331): type 1 sets the joint
        torques (World::mJointTorque), type 2 goes through the muscle
        front-end, type 3 sets each pneumatic spring's activation directly."""
        k = 0
        for o in self.mDfobjs:
            n = o.mActions.size
            if n and o.body.actuator_type == 1:
                o.torques = np.asarray(tau[k:k + n], np.float64).copy()
                o.mActions = o.torques.copy()
                self.mSoftWorld.mJointTorque = o.torques.copy()
            elif n and o.body.actuator_type == 2:
                t = torch.as_tensor(np.asarray(tau[k:k + n], np.float64))
                o.levels = o.activation_from_actions(t, self.mPhase, torch.as_tensor(o.levels)).numpy()
                o.mActions = np.asarray(tau[k:k + n], np.float64).copy()
            elif n and o.body.actuator_type == 3:
                o.pneumatic_levels = np.asarray(tau[k:k + n], np.float64).copy()
                o.mActions = o.pneumatic_levels.copy()
            k += n

    def IncPhase(self) -> None:
        self.mPhase += 1

    def Reset(self) -> None:
        for o in self.mDfobjs:
            o.levels[:] = 0.0
            o.pneumatic_levels[:] = 1.0
            o.torques[:] = 0.0
        if self.scene.n_joint_state:
            self.scene.set_joint_state(self._jq0, self._jq0)
            self.mSoftWorld.mJointQ = self._jq0.copy()
            self.mSoftWorld.mJointQd = self._jq0.copy()
        self.mPhase = 0
        self.mSoftWorld.mX = self.desc.x0.reshape(-1).copy()
        self.mSoftWorld.mV[:] = 0.0

    def SaveObj(self, filename: str, x) -> None:
        """Environment::SaveObj: one OBJ per body (vertices + surface faces),
        written asynchronously by the engine's OBJ writer (x: numpy, or a CUDA
        tensor produced on this scene's stream); FlushObj waits for the files."""
        if self._obj is None:
            bodies = []
            for i, b in enumerate(self.loaded.bodies):
                tag = "_DfObj" if b.kind == "mesh" else "_DfCloths"
                idx = i if b.kind == "mesh" else i - len(self.mDfobjs)
                faces = b.contours if b.contours is not None else np.zeros((0, 3), np.int32)
                bodies.append((b.n, faces, f"{tag}{idx}.obj"))
            self._obj = ObjWriter(bodies)
        if _is_cuda(x):
            self._obj.write(filename, x, scene=self.scene)
        else:
            self._obj.write(filename, np.asarray(x, np.float64).reshape(-1))

    def FlushObj(self) -> None:
        if self._obj is not None:
            self._obj.flush()


def init_env(total_step: int, config_path: str, device: int = 0) -> Environment:
    return Environment(loader.load_scene(config_path, total_step), device=device)


def forward_act(q, qd, jq, jqd, tau, env: Environment, is_act: bool):
    if is_act:
        env.SetActions(np.asarray(tau, np.float64))
        env.IncPhase()
    act = env.segment_activations()
    _set_joints(env, jq, jqd)
    x, v = env.scene.forward(np.asarray(q, np.float64), np.asarray(qd, np.float64), n_steps=1,
                             act=act.reshape(1, -1) if act.size else None)
    env.mSoftWorld.mX, env.mSoftWorld.mV = x.copy(), v.copy()
    njq, njqd = env.scene.joint_state()
    env.mSoftWorld.mJointQ, env.mSoftWorld.mJointQd = njq.copy(), njqd.copy()
    return [x, v, njq, njqd]


def _set_joints(env: Environment, jq, jqd) -> None:
    """Environment::Step writes jq / jqd into World::mJointQ / mJointQd before
    stepping (sim/Environment.h:278-279); empty arrays keep the current state."""
    jq = np.asarray(jq, np.float64).reshape(-1)
    jqd = np.asarray(jqd, np.float64).reshape(-1)
    if env.scene.n_joint_state and jq.size:
        env.scene.set_joint_state(jq, jqd)


def backward_act(q, qd, jq, jqd, tau, dldq, dldqd, dldjq, dldjqd, env: Environment, is_act: bool):
    with torch.enable_grad():  # also when called from an autograd backward (grad mode off there)
        return _backward_act(q, qd, jq, jqd, tau, dldq, dldqd, dldjq, dldjqd, env, is_act)


def _channels_t(env: Environment, tau_t, is_act: bool):
    """The step's activation channels as a torch vector, differentiable in
    tau through the actuator front-ends (types 1, 2 and 3)."""
    out = torch.as_tensor(env.segment_activations()).clone()
    k = 0
    for o in env.mDfobjs:
        n = o.mActions.size
        b = o.body
        if is_act and n and b.actuator_type == 1:
            out = torch.cat([out[:b.torque_offset], tau_t[k:k + n], out[b.torque_offset + n:]])
        elif is_act and n and b.actuator_type == 2:
            lv = o.activation_from_actions(tau_t[k:k + n], env.mPhase, torch.as_tensor(o.levels)).reshape(-1)
            lv = lv[: b.n_segments]
            out = torch.cat([out[:b.seg_offset], lv, out[b.seg_offset + lv.numel():]])
        elif is_act and n and b.actuator_type == 3:
            out = torch.cat([out[:b.pneumatic_offset], tau_t[k:k + n], out[b.pneumatic_offset + n:]])
        k += n
    return out


def _backward_act(q, qd, jq, jqd, tau, dldq, dldqd, dldjq, dldjqd, env: Environment, is_act: bool):
    tau_t = torch.tensor(np.asarray(tau, np.float64), requires_grad=True)
    chan = _channels_t(env, tau_t, is_act)
    if is_act:
        env.mPhase += 1
    act_np = chan.detach().numpy()
    _set_joints(env, jq, jqd)
    env.scene.forward(np.asarray(q, np.float64), np.asarray(qd, np.float64), n_steps=1,
                      act=act_np.reshape(1, -1) if act_np.size else None)
    nq = env.scene.n_joint_state
    gj = (np.asarray(dldjq, np.float64).reshape(-1), np.asarray(dldjqd, np.float64).reshape(-1)) \
        if nq and np.asarray(dldjq).size else (None, None)
    g = env.scene.backward(np.asarray(dldq, np.float64), np.asarray(dldqd, np.float64), *gj)
    dtau = np.zeros(len(tau))
    if is_act and chan.requires_grad and g["act"].size:
        (gt,) = torch.autograd.grad(chan, tau_t, torch.as_tensor(g["act"][0]), allow_unused=True)
        if gt is not None:
            dtau = gt.numpy()
    return [g["x"], g["v"], g.get("jq", np.zeros(0)), g.get("jqd", np.zeros(0)), dtau]


def forward_all(q, qd, tau, env: Environment, write_obj: Optional[str] = None):
    """Global E = tau[0], nu = tau[1] on every tet (pydifem.cc:207-221), then
    total_step steps.  write_obj: optional prefix for per-step OBJ output."""
    tau = np.asarray(tau, np.float64)
    T = env.desc.n_tets
    env._E = np.full(T, tau[0])
    env._nu = np.full(T, tau[1])
    env.scene.set_materials(env._E, env._nu)
    n = env.total_step
    x, v, traj = env.scene.forward(np.asarray(q, np.float64), np.asarray(qd, np.float64), n_steps=n, traj=True)
    if write_obj:
        os.makedirs(os.path.dirname(write_obj) or ".", exist_ok=True)
        for s in range(n):
            env.SaveObj(f"{write_obj}{s:03d}", traj[s])
        env.FlushObj()
    env.mSoftWorld.mX, env.mSoftWorld.mV = x.copy(), v.copy()
    return [x, v]


def backward_all(q, qd, tau, dldq, dldqd, env: Environment):
    g = env.scene.backward(np.asarray(dldq, np.float64), np.asarray(dldqd, np.float64))
    dtau = np.zeros(len(tau))
    dtau[0] = float(np.sum(g["E"]))
    if len(tau) > 1:
        dtau[1] = float(np.sum(g["nu"]))
    env.Reset()
    return [g["x"], g["v"], dtau]
