"""The adjoint through its two front-ends on the GPU: the torch.autograd bridge and the friction
minimisation (the reference's swSpE_minimize loop), on a twin experiment."""
import importlib

import numpy as np
import pytest

from tests.conftest import load_pkg

pytestmark = pytest.mark.gpu

N_STEPS = 80


@pytest.fixture(scope="module")
def pkg():
    p = load_pkg()
    p.build.build()
    return p


def _twin(pkg, scheme="godunov", n_cells=3000, n_gauges=60, obs_every=5):
    case = pkg.workloads.dam_break(n_cells=n_cells, scheme=scheme, friction="manning")
    model = pkg.SpModel(case)
    assert model.record(N_STEPS, 20) == N_STEPS
    x, y = case.mesh.cell_x, case.mesh.cell_y
    n_true = 0.03 * (1.0 + 0.2 * np.sin(2 * np.pi * x / 100.0) * np.cos(2 * np.pi * y / 40.0))
    rng = np.random.default_rng(11)
    cells = np.sort(rng.choice(case.mesh.cell_nb, size=n_gauges, replace=False))
    steps = np.arange(obs_every, N_STEPS + 1, obs_every)
    n_b = model.get_param("friction_1")
    model.set_param("friction", n_true)
    h_obs = model.replay_sample(cells, steps)
    model.set_param("friction", n_b)
    model.set_observations(cells, steps, h_obs)
    return model, case, n_b, n_true


def test_autograd_bridge_matches_the_adjoint(pkg):
    torch = pytest.importorskip("torch")
    ag = importlib.import_module(pkg.__name__ + ".autograd")
    model, case, n_b, _ = _twin(pkg, scheme="muscl_evr")
    h0, q0, r0 = (torch.tensor(a, requires_grad=True) for a in (case.h0, np.zeros(case.mesh.cell_nb),
                                                                np.zeros(case.mesh.cell_nb)))
    n1 = torch.tensor(n_b, requires_grad=True)
    n2 = torch.tensor(n_b, requires_grad=True)
    zb = torch.tensor(case.mesh.cell_z_b, requires_grad=True)
    J = ag.replay_cost(model, friction_1=n1, friction_2=n2, z_b=zb, h0=h0, q0=q0, r0=r0)
    (2.0 * J).backward()
    J_ref, g = model.adjoint()
    assert float(J) == J_ref
    for t, name in ((n1, "friction_1"), (n2, "friction_2"), (zb, "z_b"), (h0, "h0"), (q0, "q0"), (r0, "r0")):
        assert np.array_equal(t.grad.numpy(), 2.0 * g[name]), name
    # only some inputs: the others keep the model's values and get no gradient
    n1.grad = None
    J2 = ag.replay_cost(model, friction_1=n1)
    J2.backward()
    assert float(J2) == J_ref and np.array_equal(n1.grad.numpy(), g["friction_1"])


@pytest.mark.parametrize("algo", ["lbfgsb", "gd"])
def test_friction_twin_experiment_descends(pkg, tmp_path, algo):
    model, case, n_b, n_true = _twin(pkg)
    A = pkg.assimilation
    prob = A.FrictionProblem(model, n_b, transform=A.ControlTransform("clamp", lo=0.005, hi=0.1), alpha_spatial=1e-3,
                             k_ref=n_true, descent_dir=str(tmp_path / "descent"))
    res = A.run_minimization(prob, max_it=8, minimize_algo=algo, step=1e-3)
    assert res["J_final"] < 0.5 * res["J_init"], res["history"]
    rows = open(tmp_path / "descent" / "descent_log.csv").read().splitlines()
    assert len(rows) == res["n_grad"] + 1
    sse = [float(r.split(",")[-1]) for r in rows[1:]]
    assert sse[-1] < sse[0]
