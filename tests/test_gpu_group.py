"""GPU tests of batched scenes and the serving loop: each scene's result is
the same alone and in the mix (within 1e-5 in positions — the float atomic
accumulation order is the only difference), graph replay equals direct
stepping, and scene removal leaves the others untouched."""

import numpy as np
import pytest

import molla_b200 as m
from molla_b200 import scenes

pytestmark = pytest.mark.gpu

TOL = 1e-5


def small_scenes():
    out = scenes.batch_scenes(count=5, seed=11, n_range=(2e3, 3e4), grid_range=(16, 40))
    return out


def alone(engine, s, steps, sort_interval=16):
    cfg = m.config_for_scene(s)
    sim = m.MpmSimulation.new(engine, cfg)
    sim.set_particles(s.positions)
    sim.set_materials(s.rows, s.ids)
    sim.set_sort_interval(sort_interval)
    sim.step_n(s.dt, steps)
    return sim.read_positions()


def test_group_scenes_match_alone(engine):
    ss = small_scenes()
    total = sum(s.n for s in ss)
    cells = sum(s.grid_size ** 3 for s in ss)
    g = m.MpmGroup(engine, 16, total, cells + 256 * len(ss))
    ids = [g.add_scene(m.config_for_scene(s), s.rows, s.positions, s.ids, s.dt) for s in ss]
    g.step(30)
    for sid, s in zip(ids, ss):
        got = g.read_positions(sid)
        ref = alone(engine, s, 30)
        assert np.abs(got - ref).max() < TOL, sid
        st = g.read_status(sid)
        assert st.completed_substeps == 30 and not st.numerical_fault


def test_group_graph_equals_direct(engine):
    ss = small_scenes()[:3]
    total = sum(s.n for s in ss)
    cells = sum(s.grid_size ** 3 for s in ss) + 1024
    a = m.MpmGroup(engine, 8, total, cells)
    b = m.MpmGroup(engine, 8, total, cells)
    ia = [a.add_scene(m.config_for_scene(s), s.rows, s.positions, s.ids, s.dt) for s in ss]
    ib = [b.add_scene(m.config_for_scene(s), s.rows, s.positions, s.ids, s.dt) for s in ss]
    for _ in range(3):
        a.step(10)
    b.step_graph(10, 3)
    for x, y in zip(ia, ib):
        assert np.abs(a.read_positions(x) - b.read_positions(y)).max() < TOL


def test_group_remove_scene_keeps_others(engine):
    ss = small_scenes()[:3]
    total = sum(s.n for s in ss)
    cells = sum(s.grid_size ** 3 for s in ss) + 1024
    g = m.MpmGroup(engine, 8, total, cells)
    ids = [g.add_scene(m.config_for_scene(s), s.rows, s.positions, s.ids, s.dt) for s in ss]
    g.step(10)
    g.remove_scene(ids[1])
    g.step(10)
    for k in (0, 2):
        assert np.abs(g.read_positions(ids[k]) - alone(engine, ss[k], 20)).max() < TOL
    # the freed slot and ranges are reusable
    sid = g.add_scene(m.config_for_scene(ss[1]), ss[1].rows, ss[1].positions, ss[1].ids, ss[1].dt)
    g.step(5)
    assert np.abs(g.read_positions(sid) - alone(engine, ss[1], 5)).max() < TOL


def test_server_results_same_alone_and_in_mix(engine):
    ss = small_scenes()
    steps = [20, 35, 10, 50, 25]
    srv = m.MpmServer(engine, hbm_budget_bytes=64 << 20, max_scenes=8)
    tickets = [srv.submit(m.config_for_scene(s), s.rows, s.positions, s.ids, s.dt, n) for s, n in zip(ss, steps)]
    for _ in range(100):
        srv.run(1, substeps_per_tick=16)
        if all(srv.poll(t)[0] == 2 for t in tickets):
            break
    stats = srv.stats()
    assert stats["completed"] == len(ss)
    assert stats["tick_ms_p50"] > 0 and stats["tick_ms_p99"] >= stats["tick_ms_p50"]
    for t, s, n in zip(tickets, ss, steps):
        state, pos = srv.poll(t)
        assert state == 2
        assert np.abs(pos - alone(engine, s, n)).max() < TOL


def test_server_admission_respects_budget(engine):
    ss = small_scenes()
    per = [s.n * (2 * 27 * 4 + 64 + 44) + ((s.grid_size ** 3 + 255) // 256 * 256) * 48 for s in ss]
    budget = 3 * max(per)
    srv = m.MpmServer(engine, hbm_budget_bytes=budget, max_scenes=8)
    tickets = [srv.submit(m.config_for_scene(s), s.rows, s.positions, s.ids, s.dt, 30) for s in ss]
    srv.run(1, substeps_per_tick=5)
    st = srv.stats()
    assert st["resident_bytes"] <= budget
    if sum(per) > budget:
        assert st["admitted"] < len(ss)
    for _ in range(200):
        srv.run(1, substeps_per_tick=5)
        assert srv.stats()["resident_bytes"] <= budget
        if srv.stats()["completed"] == len(ss):
            break
    assert srv.stats()["completed"] == len(ss)
    for t in tickets:
        assert srv.poll(t)[0] == 2


def test_deterministic_group_bit_identical_alone_and_in_mix(engine):
    """Fixed-order P2G: a scene's state is bit-identical alone and in a mix,
    and from run to run (fixed_order_public_lifecycle_repeatability,
    crates/molla-solvers/tests/mpm_fixed_order_runtime.rs:65-159)."""
    ss = small_scenes()
    total = sum(s.n for s in ss)
    cells = sum(s.grid_size ** 3 for s in ss) + 256 * len(ss)

    def run(indices, repeat_tag):
        g = m.MpmGroup(engine, 16, total, cells)
        g.set_deterministic(True)
        ids = {i: g.add_scene(m.config_for_scene(ss[i]), ss[i].rows, ss[i].positions, ss[i].ids, ss[i].dt)
               for i in indices}
        g.step(12)
        g.step_graph(6, 2)
        out = {i: g.read_positions(sid) for i, sid in ids.items()}
        st = {i: g.read_status(sid) for i, sid in ids.items()}
        g.close()
        return out, st

    mix, st_mix = run(range(len(ss)), "mix")
    again, _ = run(range(len(ss)), "again")
    for i in range(len(ss)):
        assert np.array_equal(mix[i], again[i]), i
        assert st_mix[i].fault_bits == 0 and st_mix[i].completed_substeps == 24
    for i in (0, 3):
        alone_pos, _ = run([i], "alone")
        assert np.array_equal(alone_pos[i], mix[i]), i
        # and within the atomic path's tolerance of the default (atomic) mode
        assert np.abs(alone_pos[i] - alone(engine, ss[i], 24)).max() < TOL


def test_autotune_keeps_state_and_picks_a_candidate(engine):
    ss = small_scenes()[:3]
    total = sum(s.n for s in ss)
    cells = sum(s.grid_size ** 3 for s in ss) + 1024
    g = m.MpmGroup(engine, 8, total, cells)
    ids = [g.add_scene(m.config_for_scene(s), s.rows, s.positions, s.ids, s.dt) for s in ss]
    g.step(5)
    before = [g.read_positions(i) for i in ids]
    chosen, timings = g.autotune(probe_substeps=8, candidates=(2, 4, 8))
    assert chosen in (2, 4, 8) and all(v > 0 for v in timings.values())
    for i, b in zip(ids, before):
        assert np.array_equal(g.read_positions(i), b)
        assert g.read_status(i).completed_substeps == 5
    g.step(5)
    for k, i in enumerate(ids):
        assert np.abs(g.read_positions(i) - alone(engine, ss[k], 10)).max() < TOL


def alone_prec(engine, s, steps, svd, sort_interval=16, deterministic=False):
    cfg = m.config_for_scene(s, svd_precision=svd)
    sim = m.MpmSimulation.new(engine, cfg)
    sim.set_particles(s.positions)
    sim.set_materials(s.rows, s.ids)
    sim.set_sort_interval(sort_interval)
    if deterministic:
        sim.prepare_deterministic_p2g()
        sim.set_deterministic_p2g(True)
    sim.step_n(s.dt, steps)
    out = sim.read_positions()
    sim.close()
    return out


def test_group_mixed_svd_precision_each_matches_alone(engine):
    """FP32-SVD and FP64-SVD scenes share a group: each SVD form runs over its
    own scenes' items, so every scene matches its own precision run alone."""
    ss = small_scenes()
    prec = [0, 1, 0, 1, 0]
    total = sum(s.n for s in ss)
    cells = sum(s.grid_size ** 3 for s in ss) + 256 * len(ss)
    g = m.MpmGroup(engine, 16, total, cells)
    ids = [g.add_scene(m.config_for_scene(s, svd_precision=p), s.rows, s.positions, s.ids, s.dt)
           for s, p in zip(ss, prec)]
    g.step(20)
    g.step_graph(10, 1)
    for sid, s, p in zip(ids, ss, prec):
        got = g.read_positions(sid)
        assert np.abs(got - alone_prec(engine, s, 30, p)).max() < TOL, (sid, p)
        assert g.read_status(sid).completed_substeps == 30
    g.close()


def test_deterministic_mixed_precision_bit_identical_alone_and_in_mix(engine):
    ss = small_scenes()
    prec = [1, 0, 1, 0, 0]
    total = sum(s.n for s in ss)
    cells = sum(s.grid_size ** 3 for s in ss) + 256 * len(ss)

    def run(indices):
        g = m.MpmGroup(engine, 16, total, cells)
        g.set_deterministic(True)
        ids = {i: g.add_scene(m.config_for_scene(ss[i], svd_precision=prec[i]), ss[i].rows, ss[i].positions,
                              ss[i].ids, ss[i].dt) for i in indices}
        g.step(9)
        g.step_graph(5, 2)
        out = {i: g.read_positions(sid) for i, sid in ids.items()}
        g.close()
        return out

    mix = run(range(len(ss)))
    for i in (0, 1):
        assert np.array_equal(run([i])[i], mix[i]), i


def test_server_mixed_precision_exact_budgets(engine):
    """Requests of both SVD forms and step counts that are not multiples of
    the tick length: each result equals the scene run alone for exactly its
    own step count (the device-side budget stops it mid-tick)."""
    ss = small_scenes()
    steps = [23, 40, 7, 33, 16]
    prec = [1, 0, 0, 1, 1]
    srv = m.MpmServer(engine, hbm_budget_bytes=64 << 20, max_scenes=8)
    tickets = [srv.submit(m.config_for_scene(s, svd_precision=p), s.rows, s.positions, s.ids, s.dt, n)
               for s, n, p in zip(ss, steps, prec)]
    for _ in range(100):
        srv.run(1, substeps_per_tick=16)
        if all(srv.poll(t)[0] == 2 for t in tickets):
            break
    assert srv.stats()["completed"] == len(ss)
    for t, s, n, p in zip(tickets, ss, steps, prec):
        state, pos = srv.poll(t)
        assert state == 2
        assert np.abs(pos - alone_prec(engine, s, n, p)).max() < TOL, (n, p)


def test_server_retires_faulted_request(engine):
    """A served request whose state is not finite (one NaN position) latches
    the numerical fault on its first substep and stands frozen on the
    device; the server retires it at the next tick as faulted (state 3) with
    its frozen positions and fault bits, counts only the substeps it
    completed, and the requests served beside it finish normally
    (mpm.wgsl:217-231 latch; MpmActiveGridStats, mpm.rs:257-283)."""
    ss = small_scenes()
    bad = ss[0]
    pos_bad = bad.positions.copy()
    pos_bad[7, 1] = np.nan
    srv = m.MpmServer(engine, hbm_budget_bytes=64 << 20, max_scenes=8)
    tb = srv.submit(m.config_for_scene(bad), bad.rows, pos_bad, bad.ids, bad.dt, 200)
    good = [srv.submit(m.config_for_scene(s), s.rows, s.positions, s.ids, s.dt, 40) for s in ss[1:3]]
    srv.run(1, substeps_per_tick=16)
    # retired at the first tick that sees the latch, not after its 200 substeps
    state, pos = srv.poll(tb)
    st = srv.ticket_status(tb)
    assert state == 3 and st.numerical_fault and st.faulted(), (state, st)
    assert st.completed_substeps <= 1, st.completed_substeps
    # frozen where the latch caught it (at most one substep of free fall)
    assert np.isnan(pos[7, 1]) and np.allclose(pos, pos_bad, rtol=0, atol=1e-5, equal_nan=True)
    for _ in range(10):
        srv.run(1, substeps_per_tick=16)
        if all(srv.poll(t)[0] == 2 for t in good):
            break
    for t, s in zip(good, ss[1:3]):
        state_g, pos_g = srv.poll(t)
        assert state_g == 2 and srv.ticket_status(t).completed_substeps == 40
        assert np.abs(pos_g - alone(engine, s, 40)).max() < TOL
    stats = srv.stats()
    assert stats["faulted"] == 1 and stats["completed"] == 2
    assert stats["particle_steps"] == bad.n * st.completed_substeps + 40 * sum(s.n for s in ss[1:3])
    srv.close()


def test_retired_scenes_leave_at_the_next_regroup(engine):
    """Retirement through the server does not regroup the pool: the
    remaining scenes keep stepping (and match their alone runs) while the
    retired scenes' slots come back for new admissions."""
    ss = small_scenes()
    srv = m.MpmServer(engine, hbm_budget_bytes=64 << 20, max_scenes=8)
    first = [srv.submit(m.config_for_scene(s), s.rows, s.positions, s.ids, s.dt, n)
             for s, n in zip(ss[:3], (8, 60, 8))]
    srv.run(1, substeps_per_tick=8)
    assert srv.poll(first[0])[0] == 2 and srv.poll(first[2])[0] == 2
    late = [srv.submit(m.config_for_scene(s), s.rows, s.positions, s.ids, s.dt, 24) for s in ss[3:]]
    for _ in range(40):
        srv.run(1, substeps_per_tick=8)
        if all(srv.poll(t)[0] == 2 for t in first + late):
            break
    assert np.abs(srv.poll(first[1])[1] - alone(engine, ss[1], 60)).max() < TOL
    for t, s in zip(late, ss[3:]):
        assert np.abs(srv.poll(t)[1] - alone(engine, s, 24)).max() < TOL


def test_records_carried_across_calls(engine):
    """A call whose state is unchanged since the last call's final gather,
    and which no regrouping opens, starts with its scatter on that gather's
    records: 24 calls of step_n(1) between regroupings run one record-only
    gather (the first call's), like one step_n(24), and end in the same
    state; with regroupings every 8 substeps, a record-only gather follows
    each regrouping that opens a call.  Every host change the records depend
    on (particle state, mass and volume, materials, dt) makes the next call
    recompute them: its state then equals a fresh simulation set up with the
    same particles."""
    s = small_scenes()[1]
    cfg = m.config_for_scene(s)

    def make(interval):
        sim = m.MpmSimulation.new(engine, cfg)
        sim.set_particles(s.positions)
        sim.set_materials(s.rows, s.ids)
        sim.set_sort_interval(interval)
        return sim

    def stages(fn):
        engine.synchronize()
        engine.reset_profile()
        engine.profile(True)
        fn()
        engine.synchronize()
        engine.profile(False)
        prof = engine.read_profile()
        return prof["StressRecord"][0], prof["ParticleOrdering"][0]

    a = make(64)
    assert stages(lambda: [a.step_n(s.dt, 1) for _ in range(24)])[0] == 1
    b = make(64)
    assert stages(lambda: b.step_n(s.dt, 24))[0] == 1
    assert np.abs(a.read_positions() - b.read_positions()).max() < TOL
    b.close()
    d = make(8)
    rec, order = stages(lambda: [d.step_n(s.dt, 1) for _ in range(24)])
    assert rec == order == 3, (rec, order)  # the calls that regrouping opens: 1, 9 and 17
    d.close()
    a.set_sort_interval(64)
    # host changes between calls: each forces one record pass
    _, F, jp = a.read_particle_state()
    assert stages(lambda: a.step_n(s.dt, 3))[0] <= 1  # a regrouping may open it (new cadence)
    assert stages(lambda: a.step_n(s.dt, 3))[0] == 0
    for change in (lambda: a.write_particle_state(F=F * np.float32(1.02)),
                   lambda: a.set_particle_mass_volume(mass=np.full(s.n, 1.5 * cfg.particle_mass, np.float32)),
                   lambda: a.set_materials(s.rows, s.ids),
                   lambda: a.step_n(0.5 * s.dt, 1)):
        change()
        assert stages(lambda: a.step_n(s.dt, 2))[0] == 1
        assert stages(lambda: a.step_n(s.dt, 2))[0] == 0
    # the state after a change matches a fresh simulation given that state
    pos, vel = a.read_positions(), a.read_velocities()
    C, F, jp = a.read_particle_state()
    F2 = (F * np.float32(1.03)).astype(np.float32)
    a.write_particle_state(F=F2)
    a.step_n(s.dt, 6)
    c = m.MpmSimulation.new(engine, cfg)
    c.set_particles(pos, vel)
    c.set_materials(s.rows, s.ids)
    c.set_particle_mass_volume(mass=np.full(s.n, 1.5 * cfg.particle_mass, np.float32))
    c.write_particle_state(C, F2, jp)
    c.set_sort_interval(8)
    c.step_n(s.dt, 6)
    assert np.abs(a.read_positions() - c.read_positions()).max() < TOL
    assert np.abs(a.read_velocities() - c.read_velocities()).max() < 1e-4 * max(1.0, np.abs(vel).max())
    a.close()
    c.close()


def test_regroup_cadence_independent_of_call_chunking(engine):
    """The regrouping cadence is carried across calls: 64 calls of
    step_n(1) regroup as often as one step_n(64) (the reference regroups on
    its own schedule inside step_n, crates/molla-solvers/src/mpm.rs:2274-2353),
    and both give the same state."""
    s = small_scenes()[1]

    def run(chunks):
        sim = m.MpmSimulation.new(engine, m.config_for_scene(s))
        sim.set_particles(s.positions)
        sim.set_materials(s.rows, s.ids)
        sim.set_sort_interval(8)
        engine.synchronize()
        engine.reset_profile()
        engine.profile(True)
        for c in chunks:
            sim.step_n(s.dt, c)
        engine.synchronize()
        engine.profile(False)
        count = engine.read_profile()["ParticleOrdering"][0]
        pos = sim.read_positions()
        sim.close()
        return count, pos

    n_one, p_one = run([64])
    n_many, p_many = run([1] * 64)
    n_mixed, p_mixed = run([5, 3, 17, 1, 30, 8])
    assert n_one == n_many == n_mixed == 8
    assert np.abs(p_one - p_many).max() < TOL and np.abs(p_one - p_mixed).max() < TOL


def test_autotune_shapes_keeps_state_and_picks_candidates(engine):
    """The shapes autotuner (interval, item size, fused or separate kernels,
    CTAs per SM) leaves the state untouched and keeps values from its
    candidate sets."""
    ss = small_scenes()[:3]
    total = sum(s.n for s in ss)
    cells = sum(s.grid_size ** 3 for s in ss) + 1024
    g = m.MpmGroup(engine, 8, total, cells)
    ids = [g.add_scene(m.config_for_scene(s), s.rows, s.positions, s.ids, s.dt) for s in ss]
    g.step(5)
    before = [g.read_positions(i) for i in ids]
    shapes, probes = g.autotune_shapes(probe_substeps=8)
    assert shapes["sort_interval"] in (8, 16, 32, 64)
    assert shapes["item_particles"] in (640, 512, 384, 256)
    assert shapes["fused"] in (0, 1)
    assert shapes["gather_ctas_per_sm"] >= 1 and shapes["scatter_ctas_per_sm"] >= 1
    knobs = {k for k, _, _ in probes}
    assert knobs == {"sort_interval", "item_particles", "fused", "gather_ctas_per_sm", "scatter_ctas_per_sm"}
    assert all(ms > 0 for _, _, ms in probes)
    assert g.shapes() == shapes
    for i, b in zip(ids, before):
        assert np.array_equal(g.read_positions(i), b)
        assert g.read_status(i).completed_substeps == 5
    g.step(5)
    for k, i in enumerate(ids):
        assert np.abs(g.read_positions(i) - alone(engine, ss[k], 10)).max() < TOL
    g.close()


@pytest.mark.parametrize("shape", [dict(item_particles=128, fused=1, gather_ctas_per_sm=1),
                                   dict(item_particles=256, fused=0, scatter_ctas_per_sm=2, sort_interval=3)])
def test_shapes_do_not_change_results(engine, shape):
    ss = small_scenes()
    total = sum(s.n for s in ss)
    cells = sum(s.grid_size ** 3 for s in ss) + 256 * len(ss)
    g = m.MpmGroup(engine, 16, total, cells)
    ids = [g.add_scene(m.config_for_scene(s), s.rows, s.positions, s.ids, s.dt) for s in ss]
    g.set_shapes(**shape)
    got = g.shapes()
    for k, v in shape.items():
        assert got[k] == v, (k, got)
    g.step(12)
    g.step_graph(6, 2)
    for sid, s in zip(ids, ss):
        assert np.abs(g.read_positions(sid) - alone(engine, s, 24)).max() < TOL
    g.close()
