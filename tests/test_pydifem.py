"""The pydifem / api_diff surface on the GPU engine (mirrors the reference's
demo call patterns, python/demo_sus.py and demo_octopus.py)."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture
def env():
    from diff_fem_b200 import loader, pydifem as pd
    L = loader.load_scene("beam_scene/beam.json", 4, data_root=GOLDEN)
    L.desc.handle_collision = False  # gradients below are checked without the contact phase
    return pd.Environment(L)


def test_init_env_with_contact():
    os.environ["DFEM_DATA_DIR"] = GOLDEN
    from diff_fem_b200 import pydifem as pd
    e = pd.init_env(4, "beam_scene/beam.json")
    q, qd = pd.forward_all(e.mSoftWorld.mX, e.mSoftWorld.mV, [5e4, 0.3], e)
    assert np.all(np.isfinite(q)) and q.reshape(-1, 3)[:, 1].min() > -0.05 - 1e-3  # ground at y = -0.05


def test_forward_act_matches_engine(env):
    from diff_fem_b200 import pydifem as pd
    q = pd.vector2double(env.mSoftWorld.mX)
    qd = pd.vector2double(env.mSoftWorld.mV)
    x, v, jq, jqd = pd.forward_act(q, qd, [], [], np.zeros(0), env, False)
    x2, v2 = env.scene.forward(np.asarray(q), np.asarray(qd), n_steps=1)
    assert np.array_equal(x, x2) and jq.size == 0
    assert np.allclose(env.mSoftWorld.mX, x)


def test_sim_act_gradient_wrt_actions(env):
    import torch
    from diff_fem_b200.api_diff import sim_act
    n_act = sum(o.mActions.size for o in env.mDfobjs)
    assert n_act > 0
    q = torch.tensor(env.mSoftWorld.mX, dtype=torch.float64, requires_grad=True)
    qd = torch.zeros_like(q, requires_grad=True)
    jq = torch.zeros(0, dtype=torch.float64)
    tau = torch.full((n_act,), 1.0, dtype=torch.float64, requires_grad=True)
    qn, qdn, _, _ = sim_act(q, qd, jq, jq, tau, env, True)
    loss = (qn.reshape(-1, 3)[:, 0] ** 2).sum()
    loss.backward()
    assert q.grad is not None and torch.isfinite(q.grad).all()
    assert tau.grad is not None and torch.isfinite(tau.grad).all()


def test_sim_act_tau_gradient_matches_central_differences(env):
    """dL/dtau through sim_act (Normalizer::NormToReal, Muscle::SetActivationLevels
    propagation, the step's activation adjoint) against central differences of
    forward_act along a random direction; the environment's phase and
    activation levels are reset before every evaluation."""
    import torch
    from diff_fem_b200 import pydifem as pd
    from diff_fem_b200.api_diff import sim_act
    n_act = sum(o.mActions.size for o in env.mDfobjs)
    phase0 = env.mPhase
    levels0 = [o.GetActivationLevelsAggregate() for o in env.mDfobjs]
    x0 = env.mSoftWorld.mX.copy()
    v0 = 0.05 * np.random.default_rng(3).standard_normal(x0.size)

    def reset():
        env.mPhase = phase0
        for o, lv in zip(env.mDfobjs, levels0):
            o.SetActivationLevelsAggregate(lv)

    def loss(tau):
        reset()
        x, _, _, _ = pd.forward_act(x0, v0, [], [], tau, env, True)
        return float((x.reshape(-1, 3)[:, 0] ** 2).sum())

    tau0 = np.random.default_rng(4).uniform(-1.0, 1.0, n_act)
    reset()
    q = torch.tensor(x0, dtype=torch.float64)
    qd = torch.tensor(v0, dtype=torch.float64)
    tau = torch.tensor(tau0, dtype=torch.float64, requires_grad=True)
    jq = torch.zeros(0, dtype=torch.float64)
    qn, _, _, _ = sim_act(q, qd, jq, jq, tau, env, True)
    (qn.reshape(-1, 3)[:, 0] ** 2).sum().backward()
    g = tau.grad.numpy()
    assert np.abs(g).max() > 0
    d = np.random.default_rng(5).standard_normal(n_act)
    eps = 1e-4
    fd = (loss(tau0 + eps * d) - loss(tau0 - eps * d)) / (2 * eps)
    assert abs(g @ d - fd) <= 1e-5 * max(abs(fd), 1e-12), (g @ d, fd)


def test_sim_all_gradient_matches_finite_difference(env):
    import torch
    from diff_fem_b200 import pydifem as pd
    from diff_fem_b200.api_diff import sim_all
    x0 = torch.tensor(env.mSoftWorld.mX, dtype=torch.float64)
    v0 = torch.zeros_like(x0)
    tau = torch.tensor([5e4, 0.3], dtype=torch.float64, requires_grad=True)
    q, qd = sim_all(x0, v0, tau, env)
    loss = q.reshape(-1, 3)[:, 1].mean()
    loss.backward()
    g = tau.grad[0].item()
    eps = 50.0
    lp = pd.forward_all(x0.numpy(), v0.numpy(), [5e4 + eps, 0.3], env)[0].reshape(-1, 3)[:, 1].mean()
    lm = pd.forward_all(x0.numpy(), v0.numpy(), [5e4 - eps, 0.3], env)[0].reshape(-1, 3)[:, 1].mean()
    fd = (lp - lm) / (2 * eps)
    assert abs(g - fd) <= 1e-4 * max(abs(fd), 1e-12)


def test_pneumatic_actions_gradient_matches_central_differences():
    """Actuator type 3 (Dfobj::SetActions sets each pneumatic spring's
    activation to its action): dL/dtau of backward_act against central
    differences of forward_act, on the beam fixture's "Volume Verts" springs."""
    from diff_fem_b200 import loader, pydifem as pd
    env = pd.Environment(loader.load_scene("beam_scene/pneumatic.json", 1, data_root=GOLDEN))
    n_act = sum(o.mActions.size for o in env.mDfobjs)
    assert n_act == env.desc.n_segments == 18
    x0 = env.mSoftWorld.mX.copy()
    v0 = 0.05 * np.random.default_rng(6).standard_normal(x0.size)
    tau0 = np.random.default_rng(7).uniform(0.7, 1.3, n_act)
    w = np.random.default_rng(8).standard_normal(x0.size)

    def loss(tau):
        x, _, _, _ = pd.forward_act(x0, v0, [], [], tau, env, True)
        return float(w @ x)

    _, _, _, _, dtau = pd.backward_act(x0, v0, [], [], tau0, w, np.zeros_like(w), [], [], env, True)
    assert np.abs(dtau).max() > 0
    d = np.random.default_rng(9).standard_normal(n_act)
    eps = 1e-6
    fd = (loss(tau0 + eps * d) - loss(tau0 - eps * d)) / (2 * eps)
    assert abs(dtau @ d - fd) <= 1e-6 * max(abs(fd), 1e-12), (dtau @ d, fd)


def test_skeleton_joint_state_through_forward_act(tmp_path):
    """Actuator type 1: forward_act takes and returns the joint state
    (jq, jqd: World::mJointQ / mJointQd) and tau are the joint torques
    (World::mJointTorque); against the oracle stepped with the same state and
    torque channel."""
    import json
    from diff_fem_b200 import loader, pydifem as pd
    from oracle import oracle as O
    src = json.load(open(os.path.join(GOLDEN, "beam_scene", "beam.json")))
    mesh = src["Meshes"][0]
    for k in ("Muscle filename", "Attach Verts", "Attach Stiffness"):
        mesh.pop(k)
    mesh["Actuator type"] = 1
    mesh["Obj filename"] = os.path.join(GOLDEN, "beam_scene", "beam_tet.obj")
    L = loader.load_scene(os.path.join(GOLDEN, "beam_scene", "beam.json"), 1, data_root=GOLDEN)
    x0 = L.desc.x0.reshape(-1, 3)
    left = [int(i) for i in np.nonzero(np.isclose(x0[:, 0], 0.0))[0]]
    mid = [int(i) for i in np.nonzero(np.isclose(x0[:, 0], 0.15))[0]]
    mesh["Bones"] = [
        {"Parent ID": -1, "Joint Type": "ALL", "Joint Pos": [0, 0, 0], "Joint Axis": [0, 0, 0], "Vertices": left},
        {"Parent ID": 0, "Joint Type": "ROTATIONAL", "Joint Pos": [0.15, 0.05, 0.05], "Joint Axis": [0, 0, 1],
         "Vertices": mid},
    ]
    src["Parameters"][0]["Handle collision"] = False
    src["Parameters"][0]["Max Iteration"] = 4  # reached in every step: a fixed map for the differences below
    src.pop("Obstacles")
    path = tmp_path / "bones.json"
    path.write_text(json.dumps(src))
    env = pd.Environment(loader.load_scene(str(path), 1, data_root=str(tmp_path)))
    assert sum(o.mActions.size for o in env.mDfobjs) == 1
    o = O.OracleScene(env.desc)
    q, qd = env.mSoftWorld.mX.copy(), env.mSoftWorld.mV.copy()
    jq, jqd = env.mSoftWorld.mJointQ.copy(), env.mSoftWorld.mJointQd.copy()
    assert jq.size == 13 and np.array_equal(jq[:9], np.eye(3).reshape(-1))
    for step in range(3):
        tau = np.array([0.3 * (step + 1)])
        q2, qd2, jq2, jqd2 = pd.forward_act(q, qd, jq, jqd, tau, env, True)
        o.set_joint_state(jq, jqd)
        r = o.forward(q, qd, n_steps=1, act=tau.reshape(1, 1))
        jo, jdo = o.joint_state()
        assert np.abs(q2 - r["x"]).max() < 1e-9 * max(1.0, np.abs(r["x"]).max())
        assert np.abs(jq2 - jo).max() < 1e-9 and np.abs(jqd2 - jdo).max() < 1e-9
        q, qd, jq, jqd = q2, qd2, jq2, jqd2
    assert abs(jq[12]) > 1e-4
    # backward_act through the links: dq, djq, djqd and the torque's dtau
    # against central differences of the oracle's step (fixed iteration count
    # of the scene: max_iterations is reached in every step here)
    rng = np.random.default_rng(5)
    n3, nq = q.size, jq.size
    dldq, dldqd = rng.standard_normal(n3), rng.standard_normal(n3)
    dldjq, dldjqd = rng.standard_normal(nq), rng.standard_normal(nq)
    tau = np.array([0.7])
    env.mPhase = 0
    dq, dqd, djq, djqd, dtau = pd.backward_act(q, qd, jq, jqd, tau, dldq, dldqd, dldjq, dldjqd, env, True)
    assert djq.size == nq and djqd.size == nq and dtau.size == 1

    def loss(qq, qqd, a, b, t):
        o.set_joint_state(a, b)
        r = o.forward(qq, qqd, n_steps=1, act=np.reshape(t, (1, 1)))
        ja, jb = o.joint_state()
        return dldq @ r["x"] + dldqd @ r["v"] + dldjq @ ja + dldjqd @ jb, r["iters"]

    _, iters = loss(q, qd, jq, jqd, tau)
    assert iters[0] == 4
    h = 1e-6
    args = (q, qd, jq, jqd, tau)
    for name, grad, k in (("q", dq, 0), ("qd", dqd, 1), ("jq", djq, 2), ("jqd", djqd, 3), ("tau", dtau, 4)):
        dirn = rng.standard_normal(np.size(args[k]))
        ap, am = list(args), list(args)
        ap[k] = np.asarray(args[k], np.float64) + h * dirn.reshape(np.shape(args[k]))
        am[k] = np.asarray(args[k], np.float64) - h * dirn.reshape(np.shape(args[k]))
        fd = (loss(*ap)[0] - loss(*am)[0]) / (2 * h)
        an = float(np.asarray(grad).reshape(-1) @ dirn)
        assert abs(fd - an) <= 1e-5 * max(abs(fd), abs(an)) + 1e-8, (name, fd, an)


def test_save_obj_from_device_and_host_states(env, tmp_path):
    """Environment::SaveObj through the asynchronous writer: a CUDA state is
    copied on the scene's stream, a host state directly; both files carry the
    reference's format."""
    import torch
    from diff_fem_b200 import pydifem as pd
    x = env.mSoftWorld.mX.copy()
    xn, _, _, _ = pd.forward_act(x, np.zeros_like(x), [], [], np.zeros(0), env, False)
    env.SaveObj(str(tmp_path / "host"), xn)
    env.SaveObj(str(tmp_path / "dev"), torch.tensor(xn, device="cuda"))
    env.FlushObj()
    a = (tmp_path / "host_DfObj0.obj").read_text()
    b = (tmp_path / "dev_DfObj0.obj").read_text()
    assert a == b and a.startswith("v ") and "\nf " in a
    X = xn.reshape(-1, 3)
    assert a.splitlines()[0] == "v %06f %06f %06f" % tuple(X[0])


def test_demo_sus_loop_through_sim_all_matches_oracle():
    """python/demo_sus.py's optimisation loop on the suspended bridge
    (tests/golden/ref_scenes/bridgesus.npz): tau = t_scale * max(tau, 0.01)
    (forward_all uses tau[0] = E and tau[1] = nu on every tet), sim_all over
    the scene's 10 steps, loss = |mean(q) - target|, loss.backward(), an Adam
    step; dL/dtau and dL/dx0 against the oracle's adjoint of the same run,
    for two optimiser steps."""
    import torch
    from diff_fem_b200 import loader, pydifem as pd, scene as S
    from diff_fem_b200.api_diff import sim_all
    from oracle import oracle as O
    d = S.load_npz(os.path.join(GOLDEN, "ref_scenes", "bridgesus.npz"))
    L = loader.LoadedScene(desc=d, bodies=[loader.Body("mesh", 0, d.n_vertices, True)], total_step=10)
    env = pd.Environment(L)
    init_x = torch.tensor(env.mSoftWorld.mX, dtype=torch.float64, requires_grad=True)
    init_v = torch.zeros_like(init_x, requires_grad=True)
    init_tau = torch.tensor([1.0, 1.0] * 4, dtype=torch.float64, requires_grad=True)
    t_scale = torch.tensor([2e5, 0.4] * 4, dtype=torch.float64)
    target = init_x.detach().reshape(-1, 3).mean(0) + torch.tensor([0.0, -0.05, 0.0], dtype=torch.float64)
    opt = torch.optim.Adam([init_tau], lr=0.2)
    x0 = init_x.detach().numpy().copy()
    N = d.n_vertices
    for it in range(2):
        opt.zero_grad()
        tau = t_scale * torch.maximum(init_tau, init_tau * 0 + 0.01)
        q, qd = sim_all(init_x, init_v, tau, env)
        loss = (q.reshape(-1, 3).mean(0) - target).norm()
        loss.backward()
        E, nu = float(tau[0]), float(tau[1])
        o = O.OracleScene(d)
        o.set_materials(np.full(d.n_tets, E), np.full(d.n_tets, nu))
        r = o.forward(x0, np.zeros_like(x0), n_steps=10)
        diff = r["x"].reshape(-1, 3).mean(0) - target.numpy()
        gq = np.tile(diff / np.linalg.norm(diff) / N, N)
        g = o.backward(gq, np.zeros_like(gq))
        assert abs(float(loss) - np.linalg.norm(diff)) <= 1e-9 * np.linalg.norm(diff)
        want = np.zeros(8)
        want[0] = g["E"].sum() * 2e5 * (1.0 if float(init_tau[0]) > 0.01 else 0.0)
        want[1] = g["nu"].sum() * 0.4 * (1.0 if float(init_tau[1]) > 0.01 else 0.0)
        got = init_tau.grad.numpy()
        assert np.abs(got - want).max() <= 1e-7 * np.abs(want).max(), (got, want)
        assert np.abs(init_x.grad.numpy() - g["x"]).max() <= 1e-7 * np.abs(g["x"]).max()
        init_x.grad = None
        opt.step()
        env.mPhase = 0
