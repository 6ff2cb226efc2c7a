"""diff_fem scene files (JSON + OBJ + muscle files) -> SceneDesc.

Follows the setup code of the reference (all setup-time, host side):
  Environment::Environment   sim/Environment.h:86-225   (Parameters, Meshes, Clothes, Obstacles)
  Dfobj::SetDfobj/Initialize sim/Dfobj.h:142-611        (tet OBJ, masses, attachments, surface, muscles,
                                                          pneumatic "Volume Verts" springs, "Bones")
  Environment "Is underwater"  sim/Environment.h:161-166,236-247 (drag faces = the meshes' contours)
  Muscle / MakeMuscles       sim/Muscle.h:59-215, sim/Dfobj.h:732-790
  Dfcloth                    sim/Dfcloth.h:120-300      (edge springs w = 200, masses 1.5 * area / 3, no gravity)
  Dfobstacle                 sim/Dfobstacle.h           (static triangle mesh, unscaled)
Keys the reference reads but ignores (Area Density, Bending, Stretching,
Friction coefficients, tolerances) are ignored here too.
"""
from __future__ import annotations

import json
import os
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from . import scene as S


class SceneFormatError(ValueError):
    """A scene file (JSON, OBJ or muscle file) that cannot be read: the message
    names the file and, for line-based files, the line."""


def _resolve(path: str, root: Optional[str]) -> str:
    if os.path.isabs(path) and os.path.exists(path):
        return path
    for base in filter(None, [root, os.environ.get("DFEM_DATA_DIR"), os.getcwd()]):
        for cand in (os.path.join(base, path.lstrip("/")), os.path.join(base, "data", path.lstrip("/"))):
            if os.path.exists(cand):
                return cand
    raise FileNotFoundError(f"scene file not found: {path} (set DFEM_DATA_DIR to the data root)")


def read_obj(path: str, scale: float = 1.0):
    """Vertices, 't' tetrahedra (0-based, OBJMesh) and 'f' triangles (1-based in the file)."""
    v, t, f = [], [], []
    with open(path) as fh:
        for ln, line in enumerate(fh, 1):
            p = line.split()
            if not p:
                continue
            try:
                if p[0] == "v":
                    v.append([float(p[1]), float(p[2]), float(p[3])])
                elif p[0] == "t":
                    t.append([int(p[1]), int(p[2]), int(p[3]), int(p[4])])
                elif p[0] == "f":
                    f.append([int(q.split("/")[0]) - 1 for q in p[1:4]])
                    if len(f[-1]) != 3:
                        raise IndexError
            except (ValueError, IndexError):
                raise SceneFormatError(f"{path}:{ln}: malformed '{p[0]}' line: {line.strip()!r}") from None
    V = np.asarray(v, np.float64).reshape(-1, 3)
    T = np.asarray(t, np.int32).reshape(-1, 4)
    F = np.asarray(f, np.int32).reshape(-1, 3)
    if V.shape[0] == 0:
        raise SceneFormatError(f"{path}: no vertices")
    if not np.all(np.isfinite(V)):
        raise SceneFormatError(f"{path}: non-finite vertex coordinates")
    for name, a in (("tet", T), ("face", F)):
        if a.size and (a.min() < 0 or a.max() >= V.shape[0]):
            raise SceneFormatError(f"{path}: {name} vertex index out of range [0, {V.shape[0]})")
    return V * scale, T, F


# ------------------------------------------------------------------- muscles ---

def _signed_volume(p0, p1, p2, p3):
    return np.dot(np.cross(p1 - p0, p2 - p0), p3 - p0) / 6.0


def _line_triangle(p0, p1, p2, s, e):  # Muscle::isLineTriangleIntersect
    if _signed_volume(s, p0, p1, p2) * _signed_volume(e, p0, p1, p2) < 0:
        a, b, c = _signed_volume(s, e, p0, p1), _signed_volume(s, e, p1, p2), _signed_volume(s, e, p2, p0)
        return (a > 0 and b > 0 and c > 0) or (a < 0 and b < 0 and c < 0)
    return False


def _in_tet(p0, p1, p2, p3, s, e):  # Muscle::isInTetra
    return (_line_triangle(p0, p1, p2, s, e) or _line_triangle(p0, p1, p3, s, e) or
            _line_triangle(p0, p2, p3, s, e) or _line_triangle(p1, p2, p3, s, e))


def fibre_segments(points: np.ndarray, n_sampling: int = 50):
    """Muscle::Muscle: cut a fibre polyline into segments of ~arc/n_sampling."""
    pts = np.asarray(points, np.float64)
    arc = np.linalg.norm(np.diff(pts, axis=0), axis=1).sum()
    samp = arc / n_sampling
    starts, ends, acc, s0 = [], [], 0.0, 0
    for i in range(len(pts) - 1):
        acc += np.linalg.norm(pts[i + 1] - pts[i])
        if acc > samp:
            starts.append(pts[s0]); ends.append(pts[i]); acc = 0.0; s0 = i
    if ends:
        ends[-1] = pts[-1]
    return list(zip(starts, ends))


def muscle_constraints_from_fibres(x0, tets, fibres, stiffness, n_sampling=50):
    """Muscle::Initialize: per segment, tets the segment passes through or whose
    centre is close (w = exp(-dist/0.005) > 0.2), plus the tets holding the
    segment's end points.  Returns (muscle_tets, fibres, k*w, segment ids, n_segments)."""
    mt, mf, mk, ms = [], [], [], []
    nseg = 0
    P = x0[tets]
    det = np.linalg.det(np.stack([P[:, 1] - P[:, 0], P[:, 2] - P[:, 0], P[:, 3] - P[:, 0]], axis=2))
    flip = det < 0
    T = tets.copy()
    T[flip, 1], T[flip, 2] = tets[flip, 2], tets[flip, 1]
    P = x0[T]
    centers = P.mean(axis=1)
    for fib in fibres:
        for (s, e) in fibre_segments(fib, n_sampling)[:n_sampling]:
            f = (e - s) / np.linalg.norm(e - s)
            v = centers - s
            tproj = v @ f
            p = s + tproj[:, None] * f
            on = np.maximum(np.linalg.norm(p - s, axis=1), np.linalg.norm(p - e, axis=1)) / np.linalg.norm(e - s) < 1.0
            dist = np.where(on, np.linalg.norm(p - centers, axis=1), 1e5)
            dist = np.minimum(dist, np.minimum(np.linalg.norm(centers - s, axis=1), np.linalg.norm(centers - e, axis=1)))
            w = np.exp(-np.abs(dist) / 0.005)
            for j in np.nonzero(w > 0.2)[0]:
                mt.append(T[j]); mf.append(f); mk.append(stiffness * w[j]); ms.append(nseg)
            near = np.nonzero(np.linalg.norm(centers - 0.5 * (s + e), axis=1) < 4 * np.linalg.norm(e - s) + 0.1)[0]
            for j in near:
                if w[j] > 0.2:
                    continue
                if _in_tet(P[j, 0], P[j, 1], P[j, 2], P[j, 3], s, e):
                    mt.append(T[j]); mf.append(f); mk.append(stiffness * w[j]); ms.append(nseg)
            nseg += 1
    if not mt:
        return np.zeros((0, 4), np.int32), np.zeros((0, 3)), np.zeros(0), np.zeros(0, np.int32), nseg
    return np.asarray(mt, np.int32), np.asarray(mf), np.asarray(mk), np.asarray(ms, np.int32), nseg


def read_muscle_file(path: str, scale: float):
    fibres, cur, cur_id = [], [], None
    with open(path) as fh:
        for ln, line in enumerate(fh, 1):
            p = line.split()
            if len(p) < 5:
                continue
            try:
                fid = int(p[0])
                pt = [float(p[2]) * scale, float(p[3]) * scale, float(p[4]) * scale]
            except ValueError:
                raise SceneFormatError(f"{path}:{ln}: malformed muscle row: {line.strip()!r}") from None
            if cur_id is not None and fid != cur_id:
                fibres.append(np.asarray(cur))
                cur = []
            cur_id = fid
            cur.append(pt)
    if cur:
        fibres.append(np.asarray(cur))
    return fibres


# -------------------------------------------------------------------- bodies ---

@dataclass
class Body:
    kind: str                 # "mesh" or "cloth"
    offset: int               # first vertex in the world
    n: int                    # vertices
    enable_gravity: bool
    actuator_type: int = 0
    n_muscles: int = 0
    segments_per_muscle: int = 50
    contours: Optional[np.ndarray] = None   # surface faces for OBJ output (local ids)
    seg_offset: int = 0
    n_pneumatic: int = 0      # pneumatic springs ("Volume Verts"), one activation channel each
    pneumatic_offset: int = 0  # first channel of the pneumatic springs
    n_segments: int = 0       # muscle segments (activation channels from seg_offset)
    n_links: int = 0          # skeleton links ("Bones"); link torques on channels
    torque_offset: int = 0    # first channel of the joint torques (links 1..n_links-1)


@dataclass
class LoadedScene:
    desc: S.SceneDesc
    bodies: List[Body] = field(default_factory=list)
    total_step: int = 1


def load_scene(config_path: str, total_step: int = 1, data_root: Optional[str] = None) -> LoadedScene:
    path = _resolve(config_path, data_root)
    try:
        with open(path) as fh:
            cfg = json.load(fh)
    except json.JSONDecodeError as ex:
        raise SceneFormatError(f"{path}: invalid JSON: {ex}") from None
    if not isinstance(cfg, dict) or not isinstance(cfg.get("Parameters"), list) or not cfg["Parameters"]:
        raise SceneFormatError(f"{path}: no \"Parameters\" list")
    if not cfg.get("Meshes") and not cfg.get("Clothes"):
        raise SceneFormatError(f"{path}: no \"Meshes\" or \"Clothes\"")
    par = cfg["Parameters"][0]
    hz = int(par.get("Simulation HZ", 200))
    xs, masses, gmask = [], [], []
    tets, E, NU = [], [], []
    av, ap, ak = [], [], []
    mt, mf, mk, ms = [], [], [], []
    spv, spw, spc, spr = [], [], [], []
    lpar, ltyp, ljnt, lax, loff, lvt, lch = [], [], [], [], [0], [], []
    cverts, cfaces, dfaces = [], [], []
    bodies: List[Body] = []
    off, nseg_total = 0, 0
    for obj in cfg.get("Meshes", []):
        scale = float(obj.get("Scale", 0.05))
        v, t, _ = read_obj(_resolve(obj["Obj filename"], data_root), scale)
        n = v.shape[0]
        Ey, nu = float(obj.get("Youngs Modulus", 2e5)), float(obj.get("Poisson Ratio", 0.4))
        mass = S.lumped_masses(v, t, float(obj.get("Mass", 10.0)), bool(obj.get("Is Mass Same", True)))
        grav = bool(int(obj.get("Enable Gravity", 1)))
        xs.append(v); masses.append(mass); gmask.append(np.full(n, 1 if grav else 0, np.uint8))
        tets.append(t + off); E.append(np.full(t.shape[0], Ey)); NU.append(np.full(t.shape[0], nu))
        if "Attach Verts" in obj:
            k = float(obj["Attach Stiffness"])
            for i in sorted(set(int(q) for q in obj["Attach Verts"])):
                if not 0 <= i < n:
                    raise SceneFormatError(f"{path}: attach vertex {i} out of range [0, {n})")
                av.append(off + i); ap.append(v[i]); ak.append(k)
        faces, cv = S.surface_of(v, t)
        cverts.extend((cv + off).tolist()); cfaces.extend((faces + off).tolist())
        dfaces.extend((faces + off).tolist())   # Dfobj::mContours (outward surface faces)
        body = Body("mesh", off, n, grav, int(obj.get("Actuator type", 0)), contours=faces, seg_offset=nseg_total)
        if "Muscle filename" in obj:
            fibres = read_muscle_file(_resolve(obj["Muscle filename"], data_root), scale)
            a, b, c, d, nseg = muscle_constraints_from_fibres(v, t, fibres, float(obj.get("Muscle Stiffness", 5e5)))
            mt.append(a + off); mf.append(b); mk.append(c); ms.append(d + nseg_total)
            body.n_muscles = len(fibres)
            body.n_segments = nseg
            nseg_total += nseg
        if "Volume Verts" in obj:
            # Dfobj.h:231-251: each polyline of "Volume Verts" becomes one
            # PneumaticConstraint per consecutive vertex pair, rest length from
            # the scaled mesh, weight = "Muscle Stiffness"; Dfobj::SetActions
            # (actuator type 3) drives each one's activation directly
            kp = float(obj.get("Muscle Stiffness", 5e5))
            body.pneumatic_offset = nseg_total
            for line in obj["Volume Verts"]:
                ids = [int(q) for q in line]
                for i0, i1 in zip(ids[:-1], ids[1:]):
                    if not (0 <= i0 < n and 0 <= i1 < n) or i0 == i1:
                        raise SceneFormatError(f"{path}: bad volume vertex pair ({i0}, {i1}) for {n} vertices")
                    spv.append((i0 + off, i1 + off)); spw.append(kp)
                    spr.append(float(np.linalg.norm(v[i0] - v[i1]))); spc.append(nseg_total)
                    nseg_total += 1
                    body.n_pneumatic += 1
        if "Bones" in obj:
            # Dfobj.h:254-288: one Link per bone; "Joint Pos" unscaled (plus the
            # mesh offset, zero here), "Joint Axis" normalised, the bone's
            # vertices rigid.  The joint torques of actuator type 1
            # (World::mJointTorque) go on one channel per non-root link.
            if lpar:
                raise SceneFormatError(f"{path}: bones on more than one mesh (one skeleton root per scene)")
            kinds = {"ALL": 2, "ROTATIONAL": 1, "PRISMATIC": 0}
            body.torque_offset = nseg_total
            for li, bone in enumerate(obj["Bones"]):
                jt = kinds.get(bone.get("Joint Type"))
                if jt is None:
                    raise SceneFormatError(f"{path}: bone {li}: unknown joint type {bone.get('Joint Type')!r}")
                lpar.append(int(bone["Parent ID"])); ltyp.append(jt)
                ljnt.append([float(q) for q in bone["Joint Pos"]]); lax.append([float(q) for q in bone["Joint Axis"]])
                ids = [int(q) for q in bone["Vertices"]]
                if any(not 0 <= q < n for q in ids):
                    raise SceneFormatError(f"{path}: bone {li}: vertex out of range [0, {n})")
                lvt.extend(q + off for q in ids); loff.append(len(lvt))
                if li > 0:
                    lch.append(nseg_total); nseg_total += 1
                else:
                    lch.append(-1)
            body.n_links = len(lpar)
        bodies.append(body)
        off += n
    for obj in cfg.get("Clothes", []):
        scale = float(obj.get("Scale", 0.05))
        v, _, f = read_obj(_resolve(obj["Obj filename"], data_root), scale)
        n = v.shape[0]
        edges = sorted({(min(a, b), max(a, b)) for tri in f for a, b in ((tri[0], tri[1]), (tri[1], tri[2]), (tri[2], tri[0]))})
        xs.append(v); masses.append(S.triangle_masses(v, f, 1.5)); gmask.append(np.zeros(n, np.uint8))
        for a, b in edges:
            spv.append((a + off, b + off)); spw.append(200.0)  # CollisionMesh::getEdgeConstraint
            spr.append(float(np.linalg.norm(v[a] - v[b]))); spc.append(-1)
        if "Attach Verts" in obj:
            k = float(obj["Attach Stiffness"])
            for i in sorted(set(int(q) for q in obj["Attach Verts"])):
                if not 0 <= i < n:
                    raise SceneFormatError(f"{path}: attach vertex {i} out of range [0, {n})")
                av.append(off + i); ap.append(v[i]); ak.append(k)
        seen = set()
        for tri in f:
            for q in tri:
                if q not in seen:
                    seen.add(q); cverts.append(int(q) + off)
        cfaces.extend((f + off).tolist())
        bodies.append(Body("cloth", off, n, False, contours=f))
        off += n
    ox, of = [], []
    for obj in cfg.get("Obstacles", []):
        v, _, f = read_obj(_resolve(obj["Obj filename"], data_root), 1.0)
        of.append(f + sum(len(q) for q in ox)); ox.append(v)
    cat = lambda L, shape, dt: np.concatenate(L).astype(dt) if L else np.zeros(shape, dt)
    desc = S.SceneDesc(
        x0=np.concatenate(xs), mass=np.concatenate(masses), gravity_mask=np.concatenate(gmask),
        tets=cat(tets, (0, 4), np.int32), youngs=cat(E, (0,), np.float64), poisson=cat(NU, (0,), np.float64),
        attach_vertex=np.asarray(av, np.int32), attach_target=np.asarray(ap, np.float64).reshape(-1, 3),
        attach_stiffness=np.asarray(ak, np.float64),
        muscle_tets=cat(mt, (0, 4), np.int32), muscle_fiber=cat(mf, (0, 3), np.float64),
        muscle_stiffness=cat(mk, (0,), np.float64), muscle_segment=cat(ms, (0,), np.int32), n_segments=nseg_total,
        spring_vertices=np.asarray(spv, np.int32).reshape(-1, 2), spring_weight=np.asarray(spw, np.float64),
        # explicit rest lengths only with pneumatic springs (otherwise the
        # engine takes getEdgeLength of x0, as before)
        spring_rest=np.asarray(spr, np.float64) if any(c >= 0 for c in spc) else None,
        spring_channel=np.asarray(spc, np.int32) if any(c >= 0 for c in spc) else None,
        link_parent=np.asarray(lpar, np.int32), link_type=np.asarray(ltyp, np.int32),
        link_joint=np.asarray(ljnt, np.float64).reshape(-1, 3), link_axis=np.asarray(lax, np.float64).reshape(-1, 3),
        link_offsets=np.asarray(loff, np.int32), link_vertices=np.asarray(lvt, np.int32),
        link_channel=np.asarray(lch, np.int32) if lch else None,
        contact_vertices=np.asarray(cverts, np.int32), contact_faces=np.asarray(cfaces, np.int32).reshape(-1, 3),
        obstacle_x=cat(ox, (0, 3), np.float64), obstacle_faces=cat(of, (0, 3), np.int32),
        time_step=1.0 / hz, max_iterations=int(par.get("Max Iteration", 30)),
        damping=float(par.get("Damping coefficient", 0.9999)),
        gravity=tuple(float(g) for g in par.get("Gravity", [0.0, 0.0, 0.0])),
        handle_collision=bool(par.get("Handle collision", False)),
        self_collision=bool(par.get("Self-collision", True)),
        alpha=float(par.get("World Alpha", 1.0)), friction=float(par.get("World Friction", 1.0)),
        obstacle_friction=1.0, name=os.path.basename(config_path),
        # Environment::Step: underwater meshes get drag and lift on their contours instead of gravity
        # (Environment.h:161-166,236-247); each mesh's faces act on its own vertices
        underwater=bool(int(par.get("Is underwater", 0))),
        drag_faces=(np.asarray(dfaces, np.int32).reshape(-1, 3) if int(par.get("Is underwater", 0))
                    else np.zeros((0, 3), np.int32)),
    )
    return LoadedScene(desc=desc, bodies=bodies, total_step=total_step)
