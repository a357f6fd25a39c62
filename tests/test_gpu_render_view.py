"""Particle render view on the GPU (crates/molla-solvers/src/mpm_render_view.rs:20-56).

The lifecycle follows the reference's `mpm_resident_particle_rendering_and_lifecycle`
(tests/mpm_render_gpu.rs:186-254) without the rasteriser: the live float4
buffer is read back through its CUDA array interface and compared with
`read_positions`, bit for bit, before and after stepping, after emptying and
after a 50k reseed that keeps the same binding.
"""

import numpy as np
import pytest

import molla_b200 as m

pytestmark = pytest.mark.gpu


def render_cfg():
    cfg = m.MpmConfig.sand()
    cfg.grid_size = 16
    cfg.grid_origin = [-1.0, -1.0, -1.0]
    cfg.cell_size = 0.125
    cfg.max_particles = 50_000
    cfg.gravity_y = 0.0
    return cfg


def live(engine, view):
    import torch
    engine.synchronize()
    if view.particle_count() == 0:
        return np.zeros((0, 4), np.float32)
    return torch.as_tensor(view, device="cuda").cpu().numpy()


def test_render_view_lifecycle(engine):
    sim = m.MpmSimulation(engine, render_cfg())
    sim.set_particles([[-0.4, -0.2, 0.0], [0.4, 0.2, 0.0]], [[0.5, 0.0, 0.0]] * 2)
    view = sim.particle_render_view(engine)
    source = view.source()
    assert view.particle_count() == 2 and view.live_position_bytes() == 32 and view.capacity == 50_000
    before = live(engine, view)
    np.testing.assert_array_equal(before[:, :3], sim.read_positions())
    assert np.all(before[:, 3] == 0.0)

    sim.step_n(0.0005, 128)
    launches = engine.launch_count
    again = sim.particle_render_view(engine)
    assert engine.launch_count == launches  # no allocation, dispatch or copy
    assert again.matches_source(source) and again.positions() == view.positions()
    after = live(engine, again)
    np.testing.assert_array_equal(after[:, :3], sim.read_positions())
    assert np.all(after[:, 0] > before[:, 0] + 0.02)  # moved in +x at 0.5 m/s for 0.064 s

    other = m.Engine(0)
    with pytest.raises(m.GpuError):
        sim.particle_render_view(other)
    other.close()

    cfg1 = render_cfg()
    cfg1.max_particles = 1
    replacement = m.MpmSimulation(engine, cfg1)
    assert not replacement.particle_render_view(engine).matches_source(source)
    replacement.close()

    sim.set_particles(np.zeros((0, 3), np.float32))
    empty = sim.particle_render_view(engine)
    assert empty.particle_count() == 0 and empty.live_position_bytes() == 0 and empty.matches_source(source)

    i = np.arange(50_000)
    pos = np.stack([((i % 100) - 49.5) / 64.0, (((i // 100) % 100) - 49.5) / 64.0, (i // 10_000) * 0.01],
                   axis=1).astype(np.float32)
    sim.set_particles(pos)
    full = sim.particle_render_view(engine)
    assert full.particle_count() == 50_000 and full.matches_source(source)
    np.testing.assert_array_equal(live(engine, full)[:, :3], pos)
    sim.close()


def test_render_view_follows_regroup_and_batches(engine):
    """Positions stay in original particle order when the particle arrays are
    physically regrouped, and a command batch re-packs the view."""
    cfg = m.MpmConfig.sand()
    sim = m.MpmSimulation(engine, cfg)
    rng = np.random.default_rng(7)
    pts = rng.uniform(-0.3, 0.3, size=(4000, 3)).astype(np.float32)
    pts[:, 1] += 0.6
    sim.set_particles(pts, rng.normal(scale=0.2, size=(4000, 3)).astype(np.float32))
    sim.set_sort_interval(2)
    view = sim.particle_render_view()
    sim.step_n(1e-4, 9)
    np.testing.assert_array_equal(live(engine, view)[:, :3], sim.read_positions())
    batch = sim.begin_command_batch()
    rec = sim.prepare_step(1e-4, 5)
    batch.encode_step(rec)
    batch.encode_step(rec)
    batch.submit()
    got = live(engine, sim.particle_render_view())
    np.testing.assert_array_equal(got[:, :3], sim.read_positions())
    assert not np.array_equal(got[:, :3], pts)
    sim.close()


def test_read_positions_into_caller_buffers(engine):
    """read_positions(out=...) fills a caller array (pageable or pinned) with
    the same values as the allocating form and rejects a wrong buffer."""
    import torch
    cfg = m.MpmConfig.sand()
    sim = m.MpmSimulation(engine, cfg)
    rng = np.random.default_rng(3)
    pts = rng.uniform(-0.2, 0.2, size=(3000, 3)).astype(np.float32)
    pts[:, 1] += 0.5
    sim.set_particles(pts)
    sim.step_n(1e-4, 7)
    ref = sim.read_positions()
    pinned = torch.empty((4000, 3), dtype=torch.float32).pin_memory().numpy()
    got = sim.read_positions(out=pinned)
    assert got.shape == (3000, 3) and np.shares_memory(got, pinned)
    np.testing.assert_array_equal(got, ref)
    np.testing.assert_array_equal(sim.read_positions(out=np.zeros((3000, 3), np.float32)), ref)
    np.testing.assert_array_equal(sim.read_velocities(out=np.zeros((3000, 3), np.float32)), sim.read_velocities())
    for bad in (np.zeros((2999, 3), np.float32), np.zeros((3000, 3), np.float64), np.zeros((3000, 4), np.float32)):
        with pytest.raises(m.SolverError):
            sim.read_positions(out=bad)
    sim.close()
