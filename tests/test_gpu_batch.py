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


def _queue_members(pkg, scheme, topo):
    """SP members of one scheme and topography discretisation, uneven sizes, every friction law,
    with and without singular head loss, one that stops early at its t_max."""
    w = pkg.workloads
    return [
        w.channel_features(n_cells=3000, scheme=scheme, topo=topo, friction="manning", head_loss=False, seed=3),
        w.channel_features(n_cells=9000, scheme=scheme, topo=topo, friction="strickler", seed=4),
        w.channel_features(n_cells=5000, scheme=scheme, topo=topo, friction="chezy", outflow="z", seed=5),
        w.channel_features(n_cells=2000, scheme=scheme, topo=topo, friction="none", t_max=1.5, seed=9),
        w.channel_features(n_cells=700, scheme=scheme, topo=topo, friction="manning", seed=11),
    ]


def _same_as_alone(alone, members):
    for a, b in zip(alone, members):
        assert a.time == b.time
        for x, y in zip(a.state(), b.state()):
            assert _bits_equal(x, y)


@pytest.mark.parametrize("scheme,topo", [("muscl_evr", "blending"), ("godunov", "discontinuous"),
                                         ("muscl_evr", "discontinuous")])
@pytest.mark.parametrize("cfg", [(0, 1024), (2, 64), (4, 333)], ids=["v0t1024", "v2t64", "v4t333"])
def test_queue_matches_members_run_alone(pkg, scheme, topo, cfg):
    """The work-queue form (one persistent kernel over (step, phase, member, tile) items): every
    member bit for bit as run alone, in chunks that end inside a 32-step launch and after a
    member has reached its t_max, for several launch variants and tile sizes."""
    cases = _queue_members(pkg, scheme, topo)
    alone = [pkg.SpModel(c) for c in cases]
    members = [pkg.SpModel(c) for c in cases]
    batch = pkg.Batch(members)
    assert batch.config["mode"] == pkg.Batch.QUEUE
    batch.configure(pkg.Batch.QUEUE, variant=cfg[0], cells_per_tile=cfg[1], edges_per_tile=cfg[1] + 17)
    assert batch.config == {"mode": 1, "variant": cfg[0], "cells_per_tile": cfg[1], "edges_per_tile": cfg[1] + 17}
    for n in (70, 45):
        done = batch.step(n)
        for i, m in enumerate(alone):
            assert m.step(n) == done[i]
    assert done[3] < 45 and done[0] == 45          # the short member stopped at its t_max
    _same_as_alone(alone, members)


def test_queue_and_branches_agree_and_switch(pkg):
    cases = _queue_members(pkg, "muscl_evr", "blending")
    alone = [pkg.SpModel(c) for c in cases]
    members = [pkg.SpModel(c) for c in cases]
    batch = pkg.Batch(members)
    batch.step(20)
    batch.configure(pkg.Batch.BRANCHES)
    assert batch.config["mode"] == pkg.Batch.BRANCHES
    batch.step(20)
    batch.configure(pkg.Batch.QUEUE)
    batch.step(20)
    for m in alone:
        m.step(60)
    _same_as_alone(alone, members)
    mixed = pkg.Batch([pkg.SpModel(pkg.workloads.dip_channel(n_cells=2000)), pkg.SpModel(cases[0])])
    assert mixed.config["mode"] == pkg.Batch.BRANCHES
    with pytest.raises(pkg.Sw2dError, match="not an SP model"):
        mixed.configure(pkg.Batch.QUEUE)


def test_queue_autotune_keeps_results(pkg):
    """sw2d_batch_autotune times the queue's variants and tile sizes on the live states, restored
    after every trial: the run continues with the same bits."""
    cases = _queue_members(pkg, "muscl_evr", "blending")
    alone = [pkg.SpModel(c) for c in cases]
    members = [pkg.SpModel(c) for c in cases]
    batch = pkg.Batch(members)
    batch.step(25)
    rep = batch.autotune(steps=3, tile_sizes=(128, 512))
    assert rep.count("/tile128=") == 5 and "chosen" in rep
    batch.step(40)
    for m in alone:
        m.step(65)
    _same_as_alone(alone, members)


def test_queue_wait_that_runs_out(pkg):
    """A wait of the work queue that runs out (a poll limit of 0: any item whose prerequisite is
    still in flight gives up) ends the launch with an error instead of hanging; every CTA leaves
    the queue.  The device stays usable: a new batch then matches its members run alone."""
    cases = [pkg.workloads.dam_break(n_cells=20000, seed_mesh=k) for k in range(3)]
    batch = pkg.Batch([pkg.SpModel(c) for c in cases])
    batch.configure(pkg.Batch.QUEUE, cells_per_tile=64, edges_per_tile=64)
    batch.set_wait_polls(0)
    with pytest.raises(pkg.Sw2dError, match="ran out"):
        batch.step(40)
    batch.close()
    alone = [pkg.SpModel(c) for c in cases]
    members = [pkg.SpModel(c) for c in cases]
    again = pkg.Batch(members)
    again.step(40)
    for m in alone:
        m.step(40)
    _same_as_alone(alone, members)


def test_save_and_restore_point(pkg):
    """sw2d_save_point / sw2d_restore_point: the steps after a restore give the bits of the steps
    after the save (the balance slots, which keep the fluxes of edges left dry, are restored with
    the state and the time)."""
    case = pkg.workloads.gaussian_bumps(n_cells=20000, mesh="delaunay", initial="dam")
    m = pkg.SpModel(case)
    m.step(10)
    m.save_point()
    m.step(37)
    first, t_first = m.state(), m.time
    m.step(5)
    m.restore_point()
    assert m.step(37) == 37 and m.time == t_first
    for x, y in zip(first, m.state()):
        assert _bits_equal(x, y)
