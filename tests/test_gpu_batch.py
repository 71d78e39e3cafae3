"""Ensembles (sw2d_batch_*): members of uneven sizes, models and options advanced by one graph
launch must give, bit for bit, what each member gives run alone; the batch adjoint likewise."""
import numpy as np
import pytest

from tests.conftest import load_pkg

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pkg():
    p = load_pkg()
    p.build.build()
    return p


def _bits_equal(a, b):
    return np.array_equal(np.asarray(a).view(np.int64), np.asarray(b).view(np.int64))


def _members(pkg):
    w = pkg.workloads
    return [
        w.dam_break(n_cells=3000, scheme="godunov"),
        w.dam_break(n_cells=9000, scheme="muscl_evr", seed_mesh=4),
        w.channel_features(n_cells=5000, scheme="muscl_evr", topo="blending", friction="manning"),
        w.channel_features(n_cells=2000, t_max=1.5, seed=9),                    # stops early at t_max
        w.dip_channel(n_cells=4000),
        w.gaussian_bumps(n_cells=6000, seed_mesh=5),
    ]


@pytest.mark.parametrize("chunks", [(100,), (70, 40)], ids=["100", "70+40"])
def test_batch_matches_members_run_alone(pkg, chunks):
    cases = _members(pkg)
    alone = [pkg.SpModel(c) for c in cases]
    members = [pkg.SpModel(c) for c in cases]
    batch = pkg.Batch(members)
    for n in chunks:
        done = batch.step(n)
        for i, m in enumerate(alone):
            assert m.step(n) == done[i]
    assert done[3] < chunks[-1]          # the short member stopped at its t_max
    for a, b in zip(alone, members):
        assert a.time == b.time
        for x, y in zip(a.state(), b.state()):
            assert _bits_equal(x, y)


def test_batch_adjoint_matches_member_adjoints(pkg):
    cases = [pkg.workloads.dam_break(n_cells=3000, scheme=s, seed_mesh=k) for k, s in
             enumerate(["godunov", "muscl_evr", "muscl_evr"])]
    members = [pkg.SpModel(c) for c in cases]
    rng = np.random.default_rng(1)
    for m in members:
        m.record(40, 8)
        cells = np.sort(rng.choice(m.n, size=16, replace=False))
        m.set_observations(cells, np.arange(5, 41, 5), rng.uniform(0.1, 1.0, (8, 16)))
    batch = pkg.Batch(members)
    res = batch.adjoint(n_threads=3)
    for m, (J, g) in zip(members, res):
        J2, g2 = m.adjoint()
        assert J == J2
        for k in g:
            assert _bits_equal(g[k], g2[k]), k


def test_batch_reports_member_error(pkg):
    good = pkg.SpModel(pkg.workloads.dam_break(n_cells=2000))
    bad = pkg.SpModel(pkg.workloads.channel_features(n_cells=3000, impervious=True, seed=7))
    batch = pkg.Batch([good, bad])
    with pytest.raises(pkg.Sw2dError) as err:
        batch.step(5)
    assert err.value.code == -4 and "member 1" in err.value.message
