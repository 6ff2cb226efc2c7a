"""Scene descriptors and builders (host side, setup time).

A :class:`SceneDesc` holds plain numpy arrays that map one-to-one onto the
C-ABI ``dfem_scene_desc`` (include/dfem.h).  The builders here generate the
synthetic workloads (cube-grid beams, the muscle star, cloth) and apply the
reference's setup rules where the engine expects precomputed inputs:

* tet meshes of regular cube grids, 5 tets per cube with alternating parity so
  neighbouring cubes share conforming faces;
* lumped masses as in diff_fem ``Dfobj::Initialize`` (sim/Dfobj.h:506-525):
  with "Is Mass Same" each vertex gets ``Mass / totvol * sum(vol/4)`` of its
  tets, otherwise ``Mass / N``.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import List, Optional, Tuple

import numpy as np

from ._capi import DFEM_PREC_FP64, SceneDescC


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


def _i32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.int32))


@dataclass
class SceneDesc:
    x0: np.ndarray                       # (N, 3)
    mass: np.ndarray                     # (N,)
    tets: np.ndarray = field(default_factory=lambda: np.zeros((0, 4), np.int32))
    youngs: np.ndarray = field(default_factory=lambda: np.zeros(0))
    poisson: np.ndarray = field(default_factory=lambda: np.zeros(0))
    gravity_mask: Optional[np.ndarray] = None
    attach_vertex: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    attach_target: np.ndarray = field(default_factory=lambda: np.zeros((0, 3)))
    attach_stiffness: np.ndarray = field(default_factory=lambda: np.zeros(0))
    muscle_tets: np.ndarray = field(default_factory=lambda: np.zeros((0, 4), np.int32))
    muscle_fiber: np.ndarray = field(default_factory=lambda: np.zeros((0, 3)))
    muscle_stiffness: np.ndarray = field(default_factory=lambda: np.zeros(0))
    muscle_segment: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    n_segments: int = 0
    spring_vertices: np.ndarray = field(default_factory=lambda: np.zeros((0, 2), np.int32))
    spring_rest: Optional[np.ndarray] = None
    spring_weight: np.ndarray = field(default_factory=lambda: np.zeros(0))
    spring_channel: Optional[np.ndarray] = None  # -1 plain, c >= 0 pneumatic (activation channel c)
    bend_offsets: np.ndarray = field(default_factory=lambda: np.zeros(1, np.int32))
    bend_vertices: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    bend_weight: np.ndarray = field(default_factory=lambda: np.zeros(0))
    contact_vertices: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    contact_faces: np.ndarray = field(default_factory=lambda: np.zeros((0, 3), np.int32))
    obstacle_x: np.ndarray = field(default_factory=lambda: np.zeros((0, 3)))
    obstacle_faces: np.ndarray = field(default_factory=lambda: np.zeros((0, 3), np.int32))
    time_step: float = 0.01
    max_iterations: int = 10
    damping: float = 0.9999
    gravity: Tuple[float, float, float] = (0.0, 0.0, 0.0)
    handle_collision: bool = False
    self_collision: bool = False
    alpha: float = 1.0
    friction: float = 1.0
    obstacle_friction: float = 1.0
    precision: int = DFEM_PREC_FP64
    checkpoint_every: int = 1
    underwater: bool = False
    drag_faces: np.ndarray = field(default_factory=lambda: np.zeros((0, 3), np.int32))
    # articulated skeleton ("Bones"): link 0 the root (joint type ALL)
    link_parent: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    link_type: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    link_joint: np.ndarray = field(default_factory=lambda: np.zeros((0, 3)))
    link_axis: np.ndarray = field(default_factory=lambda: np.zeros((0, 3)))
    link_offsets: np.ndarray = field(default_factory=lambda: np.zeros(1, np.int32))
    link_vertices: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    link_channel: Optional[np.ndarray] = None
    name: str = "scene"

    @property
    def n_vertices(self) -> int:
        return int(np.asarray(self.x0).reshape(-1, 3).shape[0])

    @property
    def n_tets(self) -> int:
        return int(np.asarray(self.tets).reshape(-1, 4).shape[0])

    def to_c(self) -> Tuple[SceneDescC, list]:
        """ctypes struct + the arrays it points into (keep them alive)."""
        keep: list = []

        def P(arr, conv, ctype):
            if arr is None:
                return None
            a = conv(arr).reshape(-1)
            keep.append(a)
            if a.size == 0:
                return None
            return a.ctypes.data_as(C.POINTER(ctype))

        d = SceneDescC()
        x0 = _f64(self.x0).reshape(-1, 3)
        d.n_vertices = x0.shape[0]
        d.x0 = P(x0, _f64, C.c_double)
        d.mass = P(self.mass, _f64, C.c_double)
        d.gravity_mask = (P(np.asarray(self.gravity_mask, np.uint8), lambda a: np.ascontiguousarray(a, np.uint8), C.c_uint8)
                          if self.gravity_mask is not None else None)
        d.n_tets = self.n_tets
        d.tets = P(self.tets, _i32, C.c_int32)
        d.youngs = P(self.youngs, _f64, C.c_double)
        d.poisson = P(self.poisson, _f64, C.c_double)
        d.n_attach = int(np.asarray(self.attach_vertex).size)
        d.attach_vertex = P(self.attach_vertex, _i32, C.c_int32)
        d.attach_target = P(self.attach_target, _f64, C.c_double)
        d.attach_stiffness = P(self.attach_stiffness, _f64, C.c_double)
        d.n_muscle = int(np.asarray(self.muscle_segment).size)
        d.muscle_tets = P(self.muscle_tets, _i32, C.c_int32)
        d.muscle_fiber = P(self.muscle_fiber, _f64, C.c_double)
        d.muscle_stiffness = P(self.muscle_stiffness, _f64, C.c_double)
        d.muscle_segment = P(self.muscle_segment, _i32, C.c_int32)
        d.n_segments = int(self.n_segments)
        d.n_springs = int(np.asarray(self.spring_weight).size)
        d.spring_vertices = P(self.spring_vertices, _i32, C.c_int32)
        d.spring_rest = P(self.spring_rest, _f64, C.c_double)
        d.spring_weight = P(self.spring_weight, _f64, C.c_double)
        d.spring_channel = P(self.spring_channel, _i32, C.c_int32)
        d.n_bending = int(np.asarray(self.bend_weight).size)
        d.bend_offsets = P(self.bend_offsets, _i32, C.c_int32)
        d.bend_vertices = P(self.bend_vertices, _i32, C.c_int32)
        d.bend_weight = P(self.bend_weight, _f64, C.c_double)
        d.n_contact_vertices = int(np.asarray(self.contact_vertices).size)
        d.contact_vertices = P(self.contact_vertices, _i32, C.c_int32)
        d.n_contact_faces = int(np.asarray(self.contact_faces).reshape(-1, 3).shape[0])
        d.contact_faces = P(self.contact_faces, _i32, C.c_int32)
        d.n_obstacle_vertices = int(np.asarray(self.obstacle_x).reshape(-1, 3).shape[0])
        d.obstacle_x = P(self.obstacle_x, _f64, C.c_double)
        d.n_obstacle_faces = int(np.asarray(self.obstacle_faces).reshape(-1, 3).shape[0])
        d.obstacle_faces = P(self.obstacle_faces, _i32, C.c_int32)
        d.time_step = float(self.time_step)
        d.max_iterations = int(self.max_iterations)
        d.damping = float(self.damping)
        for c in range(3):
            d.gravity[c] = float(self.gravity[c])
        d.handle_collision = int(bool(self.handle_collision))
        d.self_collision = int(bool(self.self_collision))
        d.alpha = float(self.alpha)
        d.friction = float(self.friction)
        d.obstacle_friction = float(self.obstacle_friction)
        d.precision = int(self.precision)
        d.underwater = int(bool(self.underwater))
        d.n_drag_faces = int(np.asarray(self.drag_faces).reshape(-1, 3).shape[0])
        d.drag_faces = P(self.drag_faces, _i32, C.c_int32)
        d.n_links = int(np.asarray(self.link_parent).size)
        d.link_parent = P(self.link_parent, _i32, C.c_int32)
        d.link_type = P(self.link_type, _i32, C.c_int32)
        d.link_joint = P(self.link_joint, _f64, C.c_double)
        d.link_axis = P(self.link_axis, _f64, C.c_double)
        d.link_offsets = P(self.link_offsets, _i32, C.c_int32)
        d.link_vertices = P(self.link_vertices, _i32, C.c_int32)
        d.link_channel = P(self.link_channel, _i32, C.c_int32)
        d.checkpoint_every = int(self.checkpoint_every)
        return d, keep


def save_npz(desc: SceneDesc, path: str) -> None:
    """Every field of a scene descriptor into one compressed .npz file."""
    import dataclasses as _dc
    out = {}
    for f in _dc.fields(desc):
        v = getattr(desc, f.name)
        if v is None:
            continue
        out[f.name] = np.asarray(v)
    np.savez_compressed(path, **out)


def load_npz(path: str) -> SceneDesc:
    """A scene descriptor written by save_npz."""
    import dataclasses as _dc
    z = np.load(path, allow_pickle=False)
    kw = {}
    for f in _dc.fields(SceneDesc):
        if f.name not in z.files:
            continue
        v = z[f.name]
        if v.ndim == 0:
            v = v.item()
            if f.name in ("handle_collision", "self_collision", "underwater"):
                v = bool(v)
        elif f.name == "gravity":
            v = tuple(float(t) for t in v)
        kw[f.name] = v
    return SceneDesc(**kw)


# ------------------------------------------------------------------ meshes ---

# 5-tet split of the unit cube; corners indexed by (i, j, k) bits.  Parity 0
# keeps the even corners as the central tet, parity 1 the odd ones, so that
# neighbouring cubes of alternating parity cut shared faces along the same diagonal.
_EVEN = [(0, 0, 0), (1, 1, 0), (1, 0, 1), (0, 1, 1)]
_ODD = [(1, 0, 0), (0, 1, 0), (0, 0, 1), (1, 1, 1)]


def _five_tets(parity: int):
    central, corners = (_EVEN, _ODD) if parity == 0 else (_ODD, _EVEN)
    tets = [list(central)]
    for c in corners:
        nb = [q for q in central if sum(abs(a - b) for a, b in zip(q, c)) == 1]
        tets.append([c] + nb)
    return tets


def cube_grid(nx: int, ny: int, nz: int, edge: float, origin=(0.0, 0.0, 0.0),
              edge_xyz: Optional[Tuple[float, float, float]] = None):
    """Vertices (N,3) and tets (T,4) of an nx x ny x nz grid of cubes, 5 tets each."""
    ex, ey, ez = edge_xyz if edge_xyz is not None else (edge, edge, edge)
    vid = lambda i, j, k: (i * (ny + 1) + j) * (nz + 1) + k
    ii, jj, kk = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), np.arange(nz + 1), indexing="ij")
    x0 = np.stack([ii.ravel() * ex, jj.ravel() * ey, kk.ravel() * ez], axis=1) + np.asarray(origin, np.float64)
    pat = [_five_tets(0), _five_tets(1)]
    tets = []
    for i in range(nx):
        for j in range(ny):
            for k in range(nz):
                for tet in pat[(i + j + k) & 1]:
                    tets.append([vid(i + a, j + b, k + c) for (a, b, c) in tet])
    return x0, np.asarray(tets, dtype=np.int32)


def tet_volumes(x0: np.ndarray, tets: np.ndarray) -> np.ndarray:
    p = x0[tets]
    return np.abs(np.einsum("ij,ij->i", p[:, 1] - p[:, 0], np.cross(p[:, 2] - p[:, 0], p[:, 3] - p[:, 0]))) / 6.0


def lumped_masses(x0: np.ndarray, tets: np.ndarray, total_mass: float, is_mass_same: bool = True) -> np.ndarray:
    """diff_fem Dfobj::Initialize mass rule (sim/Dfobj.h:506-525)."""
    n = x0.shape[0]
    if not is_mass_same:
        return np.full(n, total_mass / n)
    vol = tet_volumes(x0, tets)
    m = np.zeros(n)
    np.add.at(m, tets.reshape(-1), np.repeat(0.25 * vol, 4))
    return total_mass / vol.sum() * m


# --------------------------------------------------------------- workloads ---

def cantilever(precision: int = DFEM_PREC_FP64) -> SceneDesc:
    """Cantilever beam: 10x4x4 cubes of 0.05 m (275 vertices, 800 tets),
    E = 1e5 Pa, nu = 0.3, 1000 kg/m^3 (20 kg, volume-lumped), x = 0 face pinned
    (25 attachments, k = 1e10), gravity -9.8, h = 1/60, 10 iterations."""
    x0, tets = cube_grid(10, 4, 4, 0.05)
    mass = lumped_masses(x0, tets, 1000.0 * 0.5 * 0.2 * 0.2, True)
    pins = np.nonzero(np.isclose(x0[:, 0], 0.0))[0].astype(np.int32)
    T = tets.shape[0]
    return SceneDesc(
        x0=x0, mass=mass, tets=tets, youngs=np.full(T, 1e5), poisson=np.full(T, 0.3),
        attach_vertex=pins, attach_target=x0[pins], attach_stiffness=np.full(pins.size, 1e10),
        time_step=1.0 / 60.0, max_iterations=10, damping=0.9999, gravity=(0.0, -9.8, 0.0),
        precision=precision, name="cantilever_10x4x4",
    )


def log_uniform_moduli(n: int, seed: int, lo: float = 1e4, hi: float = 1e6) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return 10.0 ** rng.uniform(np.log10(lo), np.log10(hi), size=n)


def inverse_stiffness(nx: int = 40, ny: int = 8, nz: int = 8, seed: int = 1234,
                      precision: int = DFEM_PREC_FP64, max_iterations: int = 20) -> SceneDesc:
    """Inverse-stiffness beam: nx x ny x nz cubes of 0.05 m (default 41x9x9 =
    3,321 vertices, 12,800 tets), per-tet E log-uniform in [1e4, 1e6] Pa from
    `seed`, nu = 0.3, 1000 kg/m^3, both x ends pinned (k = 1e10), gravity,
    h = 1/100, 20 iterations."""
    x0, tets = cube_grid(nx, ny, nz, 0.05)
    mass = lumped_masses(x0, tets, 1000.0 * nx * ny * nz * 0.05 ** 3, True)
    xmax = x0[:, 0].max()
    pins = np.nonzero(np.isclose(x0[:, 0], 0.0) | np.isclose(x0[:, 0], xmax))[0].astype(np.int32)
    T = tets.shape[0]
    return SceneDesc(
        x0=x0, mass=mass, tets=tets, youngs=log_uniform_moduli(T, seed), poisson=np.full(T, 0.3),
        attach_vertex=pins, attach_target=x0[pins], attach_stiffness=np.full(pins.size, 1e10),
        time_step=1.0 / 100.0, max_iterations=max_iterations, damping=0.9999, gravity=(0.0, -9.8, 0.0),
        precision=precision, name=f"inverse_stiffness_{nx}x{ny}x{nz}",
    )


# ------------------------------------------------------------------ muscles ---

def _point_segment_distance(p: np.ndarray, a: np.ndarray, b: np.ndarray) -> np.ndarray:
    ab = b - a
    t = np.clip(((p - a) @ ab) / max(ab @ ab, 1e-300), 0.0, 1.0)
    return np.linalg.norm(p - (a + t[:, None] * ab), axis=1)


def muscle_constraints(x0: np.ndarray, tets: np.ndarray, segments, stiffness: float,
                       weight_scale: float = 0.005, radius: Optional[float] = None):
    """Muscle constraints for fibre segments [(start, end), ...] following the
    rule of diff_fem ``Muscle::Initialize`` (sim/Muscle.h:109-215): every tet the
    segment passes through, or whose centre lies close enough that
    w = exp(-dist / 0.005) > 0.2, gets a LinearMuscleConstraint with fibre
    direction (end - start)/|end - start| and stiffness k_m * w.  Here "passes
    through" is taken as: centre within `radius` (default: half the mean edge)
    of the segment.  Returns (tets, fibres, stiffness, segment ids)."""
    centers = x0[tets].mean(axis=1)
    if radius is None:
        e = np.linalg.norm(x0[tets[:, 1]] - x0[tets[:, 0]], axis=1).mean()
        radius = 0.5 * e
    mt, mf, mk, ms = [], [], [], []
    for q, (a, b) in enumerate(segments):
        a = np.asarray(a, np.float64)
        b = np.asarray(b, np.float64)
        f = (b - a) / np.linalg.norm(b - a)
        dist = _point_segment_distance(centers, a, b)
        w = np.exp(-np.abs(dist) / weight_scale)
        sel = np.nonzero((dist < radius) | (w > 0.2))[0]
        for t in sel:
            mt.append(tets[t]); mf.append(f); mk.append(stiffness * max(w[t], 1e-3)); ms.append(q)
    if not mt:
        return (np.zeros((0, 4), np.int32), np.zeros((0, 3)), np.zeros(0), np.zeros(0, np.int32))
    return (np.asarray(mt, np.int32), np.asarray(mf), np.asarray(mk), np.asarray(ms, np.int32))


def muscle_beam(nx: int = 8, ny: int = 3, nz: int = 3, n_chains: int = 2, n_seg: int = 3,
                stiffness: float = 5e3, precision: int = DFEM_PREC_FP64) -> SceneDesc:
    """Small muscle-driven beam (parity cases): fibre chains along x, left end pinned."""
    edge = 0.05
    x0, tets = cube_grid(nx, ny, nz, edge)
    mass = lumped_masses(x0, tets, 1000.0 * nx * ny * nz * edge ** 3, True)
    L = nx * edge
    segs = []
    for c in range(n_chains):
        y = edge * (0.5 + (c % ny)) if ny > 1 else 0.5 * edge
        z = edge * (0.5 + ((c // ny) % nz)) if nz > 1 else 0.5 * edge
        for s in range(n_seg):
            segs.append(((L * s / n_seg, y, z), (L * (s + 1) / n_seg, y, z)))
    mt, mf, mk, ms = muscle_constraints(x0, tets, segs, stiffness)
    pins = np.nonzero(np.isclose(x0[:, 0], 0.0))[0].astype(np.int32)
    T = tets.shape[0]
    return SceneDesc(
        x0=x0, mass=mass, tets=tets, youngs=np.full(T, 5e4), poisson=np.full(T, 0.3),
        attach_vertex=pins, attach_target=x0[pins], attach_stiffness=np.full(pins.size, 1e8),
        muscle_tets=mt, muscle_fiber=mf, muscle_stiffness=mk, muscle_segment=ms, n_segments=len(segs),
        time_step=1.0 / 60.0, max_iterations=15, damping=0.9999, gravity=(0.0, -9.8, 0.0),
        precision=precision, name=f"muscle_beam_{nx}x{ny}x{nz}",
    )


def pneumatic_beam(nx: int = 8, ny: int = 3, nz: int = 3, stiffness: float = 1e5, muscle_segments: int = 2,
                   precision: int = DFEM_PREC_FP64) -> SceneDesc:
    """Small beam driven by pneumatic springs (actuator type 3 of Dfobj.h:
    "Volume Verts" polylines, one PneumaticConstraint per consecutive vertex
    pair, weight = "Muscle Stiffness", each on its own activation channel),
    plus one muscle chain so that muscle segments (channels 0..) and
    pneumatic springs (the channels after them) share one activation row.
    Left end pinned."""
    edge = 0.05
    x0, tets = cube_grid(nx, ny, nz, edge)
    mass = lumped_masses(x0, tets, 1000.0 * nx * ny * nz * edge ** 3, True)
    L = nx * edge
    segs = [((L * s / muscle_segments, 0.5 * edge, 0.5 * edge), (L * (s + 1) / muscle_segments, 0.5 * edge, 0.5 * edge))
            for s in range(muscle_segments)]
    mt, mf, mk, ms = muscle_constraints(x0, tets, segs, 5e3) if muscle_segments else (
        np.zeros((0, 4), np.int32), np.zeros((0, 3)), np.zeros(0), np.zeros(0, np.int32))
    # polylines along x on the top face (two rows) and the bottom face (one row)
    lines = []
    for (yv, zv) in ((ny * edge, 0.0), (ny * edge, nz * edge), (0.0, nz * edge)):
        on = np.nonzero(np.isclose(x0[:, 1], yv) & np.isclose(x0[:, 2], zv))[0]
        lines.append(on[np.argsort(x0[on, 0])])
    spv, spr, spc = [], [], []
    ch = len(segs)
    for line in lines:
        for i0, i1 in zip(line[:-1], line[1:]):
            spv.append((i0, i1)); spr.append(float(np.linalg.norm(x0[i0] - x0[i1]))); spc.append(ch)
            ch += 1
    pins = np.nonzero(np.isclose(x0[:, 0], 0.0))[0].astype(np.int32)
    T = tets.shape[0]
    return SceneDesc(
        x0=x0, mass=mass, tets=tets, youngs=np.full(T, 5e4), poisson=np.full(T, 0.3),
        attach_vertex=pins, attach_target=x0[pins], attach_stiffness=np.full(pins.size, 1e8),
        muscle_tets=mt, muscle_fiber=mf, muscle_stiffness=mk, muscle_segment=ms, n_segments=ch,
        spring_vertices=np.asarray(spv, np.int32), spring_rest=np.asarray(spr), spring_weight=np.full(len(spv), stiffness),
        spring_channel=np.asarray(spc, np.int32),
        time_step=1.0 / 60.0, max_iterations=15, damping=0.9999, gravity=(0.0, -9.8, 0.0),
        precision=precision, name=f"pneumatic_beam_{nx}x{ny}x{nz}",
    )


def articulated_beam(nx: int = 8, ny: int = 2, nz: int = 2, gravity=(0.0, -9.8, 0.0), torques: bool = True,
                     precision: int = DFEM_PREC_FP64) -> SceneDesc:
    """Small beam with an articulated skeleton (Link tree of Dfobj.h "Bones"):
    the root (joint type ALL) holds the left face, a ROTATIONAL link (axis z,
    joint at the middle face's centre) the middle face, and a PRISMATIC link
    (axis x, child of the rotational one) the right face; the two non-root
    links' joint torques are activation channels 0 and 1."""
    edge = 0.05
    x0, tets = cube_grid(nx, ny, nz, edge)
    mass = lumped_masses(x0, tets, 1000.0 * nx * ny * nz * edge ** 3, True)
    L = nx * edge
    faces = [np.nonzero(np.isclose(x0[:, 0], xv))[0].astype(np.int32) for xv in (0.0, edge * (nx // 2), L)]
    joints = np.array([[0.0, 0.0, 0.0], [edge * (nx // 2), 0.5 * ny * edge, 0.5 * nz * edge], [L, 0.5 * ny * edge, 0.5 * nz * edge]])
    T = tets.shape[0]
    return SceneDesc(
        x0=x0, mass=mass, tets=tets, youngs=np.full(T, 5e4), poisson=np.full(T, 0.3),
        n_segments=2 if torques else 0,
        link_parent=np.array([-1, 0, 1], np.int32), link_type=np.array([2, 1, 0], np.int32),
        link_joint=joints, link_axis=np.array([[0.0, 0.0, 0.0], [0.0, 0.0, 1.0], [1.0, 0.0, 0.0]]),
        link_offsets=np.cumsum([0] + [f.size for f in faces]).astype(np.int32),
        link_vertices=np.concatenate(faces), link_channel=np.array([-1, 0, 1], np.int32) if torques else None,
        time_step=1.0 / 100.0, max_iterations=20, damping=0.9999, gravity=gravity,
        precision=precision, name=f"articulated_beam_{nx}x{ny}x{nz}",
    )


def cell_mesh(cells, ex: float, ey: float, ez: float):
    """Conforming tet mesh of a set of unit cells (i, j, k) of a global grid,
    5 tets per cell with the parity of the global index (neighbouring cells
    share faces).  Returns (x0 (N,3), tets (T,4))."""
    vid = {}
    xs = []

    def v(i, j, k):
        key = (i, j, k)
        if key not in vid:
            vid[key] = len(xs)
            xs.append((i * ex, j * ey, k * ez))
        return vid[key]

    pat = [_five_tets(0), _five_tets(1)]
    tets = []
    for (i, j, k) in sorted(cells):
        for tet in pat[(i + j + k) & 1]:
            tets.append([v(i + a, j + b, k + c) for (a, b, c) in tet])
    return np.asarray(xs, np.float64), np.asarray(tets, np.int32)


def star_cells(refine: int = 2):
    """Cells of the 8-arm star: a central 6x6x3 cube block (x, z horizontal, y
    up) and two 12x2x2 arms leaving each of its four sides, in units of the
    0.05 m cube; x and z are refined `refine` times.  Returns (cells, arms)
    with arms[a] = (axis, sign, lateral cell range, length in cells)."""
    r = refine
    C, L, W, H = 6 * r, 12 * r, 2 * r, 2   # centre width, arm length, arm width (cells)
    cells = {(i, j, k) for i in range(C) for j in range(3) for k in range(C)}
    arms = []
    for axis in (0, 2):
        for sign in (-1, 1):
            for lat0 in (0, C - W):            # two arms per side, flush with the side's ends
                arms.append((axis, sign, (lat0, lat0 + W), L))
                for a in range(L):
                    o = C + a if sign > 0 else -1 - a
                    for lat in range(lat0, lat0 + W):
                        for j in range(H):
                            cells.add((o, j, lat) if axis == 0 else (lat, j, o))
    return cells, arms


def muscle_star(refine: int = 2, chains_per_arm: int = 8, seg_per_chain: int = 6, stiffness: float = 5e3,
                youngs: float = 5e4, ground: bool = True, mu: float = 0.5,
                precision: int = DFEM_PREC_FP64) -> SceneDesc:
    """Muscle star: a central 6x6x3 block of 0.05 m cubes with 8 arms of 12x2x2
    cubes (two per side), x and z refined `refine` times (refine=2: 0.025 m x
    0.05 m x 0.025 m cells, 1,968 cells, 9,840 tets; refine=1: 2,460 tets).
    `chains_per_arm` fibre chains run along every arm (one per cross-section
    cell for refine=2: 64 chains), each split into `seg_per_chain` segments
    (384 segments); muscle stiffness 5e3.  With `ground`, an obstacle quad lies
    1e-3 below the body with friction `mu`.  h = 1/60, 15 iterations."""
    ex, ey, ez = 0.05 / refine, 0.05, 0.05 / refine
    cells, arms = star_cells(refine)
    x0, tets = cell_mesh(cells, ex, ey, ez)
    vol = tet_volumes(x0, tets).sum()
    mass = lumped_masses(x0, tets, 1000.0 * vol, True)
    C = 6 * refine
    segs = []
    for (axis, sign, (l0, l1), L) in arms:
        lats = [(l0 + a + 0.5) for a in range(l1 - l0)]
        heights = [0.5, 1.5]
        spots = [(lat, h) for h in heights for lat in lats][:chains_per_arm]
        start = C if sign > 0 else 0
        for (lat, h) in spots:
            for q in range(seg_per_chain):
                a0 = start + sign * L * q / seg_per_chain
                a1 = start + sign * L * (q + 1) / seg_per_chain
                if axis == 0:
                    p0, p1 = (a0 * ex, h * ey, lat * ez), (a1 * ex, h * ey, lat * ez)
                else:
                    p0, p1 = (lat * ex, h * ey, a0 * ez), (lat * ex, h * ey, a1 * ez)
                segs.append((p0, p1))
    mt, mf, mk, ms = muscle_constraints(x0, tets, segs, stiffness, radius=0.5 * min(ex, ey, ez))
    T = tets.shape[0]
    kw = {}
    if ground:
        faces, cverts = surface_of(x0, tets)
        ctr = x0.mean(axis=0)
        gx, gf = ground_quad(x0[:, 1].min() - 1e-3, 2.0, center=(ctr[0], ctr[2]))
        kw = dict(contact_vertices=cverts, contact_faces=faces, obstacle_x=gx, obstacle_faces=gf,
                  handle_collision=True, obstacle_friction=mu)
    return SceneDesc(
        x0=x0, mass=mass, tets=tets, youngs=np.full(T, youngs), poisson=np.full(T, 0.3),
        muscle_tets=mt, muscle_fiber=mf, muscle_stiffness=mk, muscle_segment=ms, n_segments=len(segs),
        time_step=1.0 / 60.0, max_iterations=15, damping=0.9999, gravity=(0.0, -9.8, 0.0),
        precision=precision, name=f"muscle_star_r{refine}", **kw,
    )


def uneven_batch(n_scenes: int = 256, seed: int = 7, t_lo: float = 1e3, t_hi: float = 5e4,
                 precision: int = DFEM_PREC_FP64, max_iterations: int = 15, ground: bool = True):
    """Batch of independent scenes of uneven size: tet counts log-uniform in
    [t_lo, t_hi] from `seed`, alternating beams (cube-grid bars as the
    cantilever / inverse-stiffness scenes, cross-section ny = nz, length 5x the
    width, x = 0 face pinned) and muscle stars, each on its own ground
    obstacle with `ground` (arm length and refinement chosen to approach the
    target count).  Per-scene log-uniform moduli in [1e4, 1e6] Pa.  All share
    h = 1/60, 15 iterations, damping 0.9999 and gravity.  Returns (descs,
    target tet counts)."""
    import dataclasses
    rng = np.random.default_rng(seed)
    targets = np.exp(rng.uniform(np.log(t_lo), np.log(t_hi), size=n_scenes))
    descs = []
    stars = {}  # the star geometry depends only on the refinement: build each once
    for q, tgt in enumerate(targets):
        if q % 2 == 0:
            w = max(2, int(round((tgt / 25.0) ** (1.0 / 3.0))))
            nx = max(2, int(round(tgt / (5.0 * w * w))))
            x0, tets = cube_grid(nx, w, w, 0.05)
            mass = lumped_masses(x0, tets, 1000.0 * nx * w * w * 0.05 ** 3, True)
            pins = np.nonzero(np.isclose(x0[:, 0], 0.0))[0].astype(np.int32)
            T = tets.shape[0]
            d = SceneDesc(
                x0=x0, mass=mass, tets=tets, youngs=log_uniform_moduli(T, 1000 + q), poisson=np.full(T, 0.3),
                attach_vertex=pins, attach_target=x0[pins], attach_stiffness=np.full(pins.size, 1e10),
                time_step=1.0 / 60.0, max_iterations=max_iterations, damping=0.9999, gravity=(0.0, -9.8, 0.0),
                precision=precision, name=f"beam_{nx}x{w}x{w}")
        else:
            refine = 1 if tgt < 2460 * 1.7 else (2 if tgt < 9840 * 1.7 else 3)
            if refine not in stars:
                stars[refine] = muscle_star(refine=refine, chains_per_arm=min(8, 4 * refine), ground=ground,
                                            precision=precision)
            base = stars[refine]
            d = dataclasses.replace(base, youngs=log_uniform_moduli(base.n_tets, 1000 + q),
                                    max_iterations=max_iterations)
        descs.append(d)
    return descs, targets


# ------------------------------------------------------------------ contact ---

def tet_surface(tets: np.ndarray):
    """Boundary triangles of a tet mesh (faces used by exactly one tet) and the
    surface vertices in first-appearance order — the contact set of diff_fem
    ``Dfobj::Initialize`` (sim/Dfobj.h:542-565), found with a hash instead of
    the reference's O(F^2) duplicate test.  Faces are oriented outward."""
    faces = {}
    for t, tet in enumerate(tets):
        for drop in range(4):
            f = tuple(int(tet[k]) for k in range(4) if k != drop)
            key = tuple(sorted(f))
            faces.setdefault(key, []).append((t, drop, f))
    tris, verts, seen = [], [], set()
    for key, lst in faces.items():
        if len(lst) != 1:
            continue
        t, drop, f = lst[0]
        tris.append((t, drop, f))
    return tris


def surface_of(x0: np.ndarray, tets: np.ndarray):
    """(surface faces (F,3) outward, contact vertices in first-appearance order)."""
    out_f, verts, seen = [], [], set()
    for t, drop, f in tet_surface(tets):
        a, b, c = f
        opp = x0[tets[t][drop]]
        n = np.cross(x0[b] - x0[a], x0[c] - x0[a])
        if np.dot(n, opp - x0[a]) > 0:
            a, b = b, a
        out_f.append((a, b, c))
        for v in (a, b, c):
            if v not in seen:
                seen.add(v)
                verts.append(v)
    return np.asarray(out_f, np.int32), np.asarray(verts, np.int32)


def underwater_block(nx: int = 4, ny: int = 2, nz: int = 3, edge: float = 0.05, speed: float = 0.6,
                     precision: int = DFEM_PREC_FP64, seed: int = 3):
    """A soft block moving through still water (underwater drag and lift on
    its outward surface faces, no gravity).  Returns (desc, initial velocity
    (N,3)): a uniform swim velocity plus a seeded per-vertex wobble."""
    x0, tets = cube_grid(nx, ny, nz, edge)
    mass = lumped_masses(x0, tets, 1000.0 * nx * ny * nz * edge ** 3, True)
    faces, _ = surface_of(x0, tets)
    T = tets.shape[0]
    d = SceneDesc(
        x0=x0, mass=mass, tets=tets, youngs=np.full(T, 3e4), poisson=np.full(T, 0.3),
        time_step=1.0 / 60.0, max_iterations=10, damping=0.9999, gravity=(0.0, -9.8, 0.0),
        underwater=True, drag_faces=faces, precision=precision, name=f"underwater_block_{nx}x{ny}x{nz}")
    rng = np.random.default_rng(seed)
    v0 = np.tile(np.array([speed, 0.25 * speed, -0.4 * speed]), (x0.shape[0], 1))
    v0 += 0.1 * speed * rng.standard_normal(v0.shape)
    return d, v0


def ground_quad(y: float, half: float, center=(0.0, 0.0)):
    """Static ground obstacle: one quad (two triangles) at height y, normal +y."""
    cx, cz = center
    xs = np.array([[cx - half, y, cz - half], [cx + half, y, cz - half], [cx + half, y, cz + half], [cx - half, y, cz + half]])
    faces = np.array([[0, 2, 1], [0, 3, 2]], np.int32)
    return xs, faces


def drop_box(nx: int = 4, ny: int = 2, nz: int = 4, height: float = 0.02, v0: float = -1.0,
             mu: float = 1.0, precision: int = DFEM_PREC_FP64) -> SceneDesc:
    """Small soft box dropped onto a ground quad (obstacle contact parity cases)."""
    edge = 0.05
    x0, tets = cube_grid(nx, ny, nz, edge, origin=(0.0, height, 0.0))
    mass = lumped_masses(x0, tets, 1000.0 * nx * ny * nz * edge ** 3, True)
    faces, cverts = surface_of(x0, tets)
    gx, gf = ground_quad(0.0, 1.0, center=(0.5 * nx * edge, 0.5 * nz * edge))
    T = tets.shape[0]
    d = SceneDesc(
        x0=x0, mass=mass, tets=tets, youngs=np.full(T, 5e4), poisson=np.full(T, 0.3),
        contact_vertices=cverts, contact_faces=faces, obstacle_x=gx, obstacle_faces=gf,
        handle_collision=True, obstacle_friction=mu,
        time_step=1.0 / 60.0, max_iterations=15, damping=0.9999, gravity=(0.0, -9.8, 0.0),
        precision=precision, name=f"drop_box_{nx}x{ny}x{nz}",
    )
    d.initial_velocity = np.tile([0.0, v0, 0.0], x0.shape[0])
    return d


def icosphere(radius: float, subdiv: int, center=(0.0, 0.0, 0.0)):
    """Triangulated sphere (icosahedron refined `subdiv` times, vertices pushed
    to the sphere), outward faces.  Returns (vertices (V,3), faces (F,3))."""
    t = (1.0 + 5 ** 0.5) / 2.0
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
         (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2), (10, 7, 6),
         (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10),
         (8, 6, 7), (9, 8, 1)]
    verts = [np.asarray(p, np.float64) / np.linalg.norm(p) for p in v]
    for _ in range(subdiv):
        mid = {}

        def midpoint(a, b):
            key = (min(a, b), max(a, b))
            if key not in mid:
                m = verts[a] + verts[b]
                verts.append(m / np.linalg.norm(m))
                mid[key] = len(verts) - 1
            return mid[key]

        nf = []
        for a, b, c in f:
            ab, bc, ca = midpoint(a, b), midpoint(b, c), midpoint(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        f = nf
    X = radius * np.asarray(verts) + np.asarray(center, np.float64)
    F = np.asarray(f, np.int32)
    # outward orientation
    c0 = np.asarray(center, np.float64)
    for k, (a, b, c) in enumerate(F):
        n = np.cross(X[b] - X[a], X[c] - X[a])
        if np.dot(n, X[a] - c0) < 0:
            F[k] = (a, c, b)
    return X, F


def cloth_on_ball(nv: int = 64, edge: float = 0.02, radius: float = 0.2, drop: float = 0.3, subdiv: int = 3,
                  stretch: float = 1e3, bend: float = 1e-3, density: float = 0.2, mu: float = 0.3,
                  precision: int = DFEM_PREC_FP64) -> SceneDesc:
    """Cloth on a ball: an nv x nv cloth (edge 0.02 m; 64x64: 7,938 triangles,
    springs on every edge, bending on every interior vertex; membrane 1e3,
    bending 1e-3, 0.2 kg/m^2, gravity on) centred `drop` m above a ball of
    radius `radius`, and a ground quad below the ball.  The ball is a static
    obstacle surface (an icosphere, `subdiv` refinements): soft-soft contact
    is not built, so the ball does not deform.  Every cloth vertex is a
    contact vertex; obstacle friction mu.  h = 1/120, 20 iterations."""
    side = (nv - 1) * edge
    x0, tris, springs, boff, bvert = cloth_grid(nv, nv, edge, origin=(-0.5 * side, radius + drop, -0.5 * side))
    mass = triangle_masses(x0, tris, density)
    bx, bf = icosphere(radius, subdiv)
    gx, gf = ground_quad(-radius - 1e-3, 2.0)
    ox = np.concatenate([bx, gx])
    of = np.concatenate([bf, gf + len(bx)]).astype(np.int32)
    return SceneDesc(
        x0=x0, mass=mass, spring_vertices=springs, spring_weight=np.full(len(springs), stretch),
        bend_offsets=boff, bend_vertices=bvert, bend_weight=np.full(len(boff) - 1, bend),
        contact_vertices=np.arange(x0.shape[0], dtype=np.int32), contact_faces=tris,
        obstacle_x=ox, obstacle_faces=of, handle_collision=True, obstacle_friction=mu,
        time_step=1.0 / 120.0, max_iterations=20, damping=0.9999, gravity=(0.0, -9.8, 0.0),
        precision=precision, name=f"cloth_on_ball_{nv}x{nv}",
    )


def cloth_on_block(nv: int = 4, edge: float = 0.014, block=(2, 1, 2), block_edge: float = 0.03, gap: float = 0.004,
                   offset=(0.0031, -0.0047),
                   v0: float = -0.6, stretch: float = 200.0, bend: float = 1e-3, density: float = 0.3,
                   block_E: float = 5e4, mu_self: float = 0.3, mu_ground: float = 0.5, alpha: float = 0.5,
                   precision: int = DFEM_PREC_FP64) -> SceneDesc:
    """Soft-soft contact case: an nv x nv cloth falling (initial velocity v0
    m/s, `gap` m above) onto a soft tet block that rests on a ground quad.
    Contact vertices are every cloth vertex and the block's surface
    vertices; contact faces are the cloth's triangles and the block's surface
    triangles; self-collision on (soft-soft friction mu_self = "World
    Friction"), obstacle friction mu_ground.  The cloth is centred over the
    block shifted by `offset` (x, z), so that no vertex lies over an edge of
    the other surface's triangles.  Contact relaxation ("World Alpha")
    `alpha`: a vertex shared by several hit faces receives every group's
    correction, and unrelaxed Jacobi sweeps (alpha = 1) can diverge on the
    larger blocks.  h = 1/120, 20 iterations."""
    nx, ny, nz = block
    bx0, btets = cube_grid(nx, ny, nz, block_edge)
    bmass = lumped_masses(bx0, btets, 1000.0 * nx * ny * nz * block_edge ** 3, True)
    bfaces, bverts = surface_of(bx0, btets)
    top = ny * block_edge
    side = (nv - 1) * edge
    cx, cz = 0.5 * nx * block_edge, 0.5 * nz * block_edge
    x0c, tris, springs, boff, bvert = cloth_grid(nv, nv, edge, origin=(cx - 0.5 * side + offset[0], top + gap,
                                                                 cz - 0.5 * side + offset[1]))
    mc = triangle_masses(x0c, tris, density)
    nc = x0c.shape[0]
    gx, gf = ground_quad(-1e-3, 1.0, center=(cx, cz))
    T = btets.shape[0]
    d = SceneDesc(
        x0=np.concatenate([x0c, bx0]), mass=np.concatenate([mc, bmass]),
        tets=btets + nc, youngs=np.full(T, block_E), poisson=np.full(T, 0.3),
        spring_vertices=springs, spring_weight=np.full(len(springs), stretch),
        bend_offsets=boff, bend_vertices=bvert, bend_weight=np.full(len(boff) - 1, bend),
        contact_vertices=np.concatenate([np.arange(nc), bverts + nc]).astype(np.int32),
        contact_faces=np.concatenate([tris, bfaces + nc]).astype(np.int32),
        obstacle_x=gx, obstacle_faces=gf, handle_collision=True, self_collision=True,
        friction=mu_self, obstacle_friction=mu_ground, alpha=alpha,
        time_step=1.0 / 120.0, max_iterations=20, damping=0.9999, gravity=(0.0, -9.8, 0.0),
        precision=precision, name=f"cloth_{nv}x{nv}_on_block_{nx}x{ny}x{nz}",
    )
    d.initial_velocity = np.concatenate([np.tile([0.0, v0, 0.0], nc), np.zeros(3 * bx0.shape[0])])
    return d


def soft_ball(radius: float, subdiv: int, center=(0.0, 0.0, 0.0), density: float = 1000.0):
    """Tet-meshed ball: one tet from the centre to every face of an icosphere
    (`subdiv` refinements: 20 * 4^subdiv tets).  Returns (vertices: surface
    then centre, tets, surface faces (outward), surface vertex ids, masses)."""
    X, F = icosphere(radius, subdiv, center)
    c = len(X)
    x0 = np.concatenate([X, np.asarray(center, np.float64)[None]])
    tets = np.concatenate([np.full((len(F), 1), c, np.int32), F], axis=1).astype(np.int32)
    mass = lumped_masses(x0, tets, density * 4.0 / 3.0 * np.pi * radius ** 3, True)
    return x0, tets, F.astype(np.int32), np.arange(c, dtype=np.int32), mass


def cloth_on_soft_ball(nv: int = 64, edge: float = 0.02, radius: float = 0.2, drop: float = 0.3, subdiv: int = 4,
                       stretch: float = 1e3, bend: float = 1e-3, density: float = 0.2, ball_E: float = 5e4,
                       mu: float = 0.3, alpha: float = 0.5, precision: int = DFEM_PREC_FP64) -> SceneDesc:
    """Cloth on a soft ball (soft-soft contact): the cloth of cloth_on_ball
    (nv x nv, edge 0.02 m, membrane 1e3, bending 1e-3, 0.2 kg/m^2, gravity on)
    centred `drop` m above a tet-meshed ball (radius 0.2 m, 20 * 4^subdiv
    tets: 5,120 at subdiv 4; E = ball_E, nu 0.3, 1000 kg/m^3, gravity on)
    that rests on a ground quad.  Self-collision on: the cloth's vertices and
    triangles and the ball's surface are the soft contact surface ("World
    Friction" mu); ground friction mu; relaxation alpha.  h = 1/120, 20
    iterations."""
    side = (nv - 1) * edge
    # the cloth's corner offset off the ball's symmetry planes
    xc, tris, springs, boff, bvert = cloth_grid(nv, nv, edge, origin=(-0.5 * side + 0.0013, radius + drop,
                                                                   -0.5 * side - 0.0021))
    mc = triangle_masses(xc, tris, density)
    xb, btets, bfaces, bsurf, mb = soft_ball(radius, subdiv)
    nc = xc.shape[0]
    gx, gf = ground_quad(-radius - 1e-3, 2.0)
    T = btets.shape[0]
    return SceneDesc(
        x0=np.concatenate([xc, xb]), mass=np.concatenate([mc, mb]),
        tets=btets + nc, youngs=np.full(T, ball_E), poisson=np.full(T, 0.3),
        spring_vertices=springs, spring_weight=np.full(len(springs), stretch),
        bend_offsets=boff, bend_vertices=bvert, bend_weight=np.full(len(boff) - 1, bend),
        contact_vertices=np.concatenate([np.arange(nc), bsurf + nc]).astype(np.int32),
        contact_faces=np.concatenate([tris, bfaces + nc]).astype(np.int32),
        obstacle_x=gx, obstacle_faces=gf, handle_collision=True, self_collision=True,
        friction=mu, obstacle_friction=mu, alpha=alpha,
        time_step=1.0 / 120.0, max_iterations=20, damping=0.9999, gravity=(0.0, -9.8, 0.0),
        precision=precision, name=f"cloth_{nv}x{nv}_on_soft_ball_{T}",
    )


# -------------------------------------------------------------------- cloth ---

def cloth_grid(nv_x: int, nv_z: int, edge: float, origin=(0.0, 0.0, 0.0)):
    """Flat cloth in the xz plane: (nv_x * nv_z) vertices, two triangles per quad
    (diagonal (i,j)-(i+1,j+1)), springs on every edge, bending stencils on every
    interior vertex (centre + 6-ring in cyclic order).  Returns
    (x0, triangles, springs, bend_offsets, bend_vertices)."""
    vid = lambda i, j: i * nv_z + j
    ii, jj = np.meshgrid(np.arange(nv_x), np.arange(nv_z), indexing="ij")
    x0 = np.stack([ii.ravel() * edge, np.zeros(ii.size), jj.ravel() * edge], axis=1) + np.asarray(origin, np.float64)
    tris, springs = [], set()
    for i in range(nv_x - 1):
        for j in range(nv_z - 1):
            a, b, c, d = vid(i, j), vid(i + 1, j), vid(i + 1, j + 1), vid(i, j + 1)
            tris.append((a, b, c)); tris.append((a, c, d))
            for e in ((a, b), (b, c), (a, c), (c, d), (d, a)):
                springs.add((min(e), max(e)))
    boff, bvert = [0], []
    for i in range(1, nv_x - 1):
        for j in range(1, nv_z - 1):
            ring = [vid(i + 1, j), vid(i + 1, j + 1), vid(i, j + 1), vid(i - 1, j), vid(i - 1, j - 1), vid(i, j - 1)]
            bvert.extend([vid(i, j)] + ring)
            boff.append(len(bvert))
    return (x0, np.asarray(tris, np.int32), np.asarray(sorted(springs), np.int32),
            np.asarray(boff, np.int32), np.asarray(bvert, np.int32))


def triangle_masses(x0: np.ndarray, tris: np.ndarray, density: float) -> np.ndarray:
    """Area-lumped cloth masses: each vertex gets density * area / 3 of its
    triangles (diff_fem Dfcloth::Initialize + CollisionMesh::getTriangleMass)."""
    p = x0[tris]
    area = 0.5 * np.linalg.norm(np.cross(p[:, 1] - p[:, 0], p[:, 2] - p[:, 0]), axis=1)
    m = np.zeros(x0.shape[0])
    np.add.at(m, tris.reshape(-1), np.repeat(density * area / 3.0, 3))
    return m


def cloth_sheet(nv: int = 8, edge: float = 0.02, stretch: float = 200.0, bend: float = 1e-3,
                density: float = 1.5, pin_corners: bool = True, precision: int = DFEM_PREC_FP64) -> SceneDesc:
    """Small hanging cloth (parity cases): springs + bending, two corners pinned."""
    x0, tris, springs, boff, bvert = cloth_grid(nv, nv, edge)
    mass = triangle_masses(x0, tris, density)
    pins = np.asarray([0, (nv - 1) * nv], np.int32) if pin_corners else np.zeros(0, np.int32)
    return SceneDesc(
        x0=x0, mass=mass, spring_vertices=springs, spring_weight=np.full(len(springs), stretch),
        bend_offsets=boff, bend_vertices=bvert, bend_weight=np.full(len(boff) - 1, bend),
        attach_vertex=pins, attach_target=x0[pins], attach_stiffness=np.full(pins.size, 1e5),
        contact_faces=tris,
        time_step=1.0 / 120.0, max_iterations=20, damping=0.9999, gravity=(0.0, -9.8, 0.0),
        precision=precision, name=f"cloth_{nv}x{nv}",
    )
