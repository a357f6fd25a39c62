// mpm_abi.cu — the extern "C" entry points declared in include/molla_mpm.h.
// Each function maps library exceptions to status codes and records the
// message for mpm_last_error on the calling thread.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "mpm_runtime.cuh"
#include "mpm_checkpoint.cuh"
#include "mpm_f64.cuh"

using mpm::Error;

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

template <class F>
int guard(F&& f) {
  try {
    f();
    g_last_error.clear();
    return MPM_OK;
  } catch (const Error& e) {
    return fail(e.code, e.what());
  } catch (const std::bad_alloc&) {
    return fail(MPM_ERR_NOMEM, "host allocation failed");
  } catch (const std::exception& e) {
    return fail(MPM_ERR_INVALID, e.what());
  }
}

#define REQUIRE(cond, code, msg) \
  do {                           \
    if (!(cond)) throw Error((code), (msg)); \
  } while (0)

bool finite3(const float* v) { return std::isfinite(v[0]) && std::isfinite(v[1]) && std::isfinite(v[2]); }

void validate_config(const mpm_config& c) {
  REQUIRE(c.grid_size > 0 && (uint64_t)c.grid_size * c.grid_size * c.grid_size < (1ull << 40), MPM_ERR_INVALID,
          "MPM grid dimensions overflow or are empty");
  REQUIRE(std::isfinite(c.cell_size) && c.cell_size > 0.f && finite3(c.grid_origin), MPM_ERR_INVALID,
          "MPM grid exceeds device capacity or has invalid spacing/origin");
  REQUIRE(c.rheology.kind <= MPM_RHEOLOGY_VISCOUS, MPM_ERR_INVALID, "unknown MPM rheology");
  REQUIRE(c.time_step <= MPM_TIME_STEP_IMPLICIT, MPM_ERR_INVALID, "unknown MPM time step");
  REQUIRE(c.walls <= MPM_WALLS_STICKY, MPM_ERR_INVALID, "unknown MPM wall model");
  REQUIRE(c.svd_precision <= MPM_SVD_FP64, MPM_ERR_INVALID, "unknown MPM SVD precision");
  REQUIRE(c.boundary_pad == 0 || c.boundary_pad * 2 < c.grid_size, MPM_ERR_INVALID, "MPM boundary pad too wide");
}

mpm_rheology sand_row(float phi) {
  mpm_rheology r{};
  r.kind = MPM_RHEOLOGY_SAND;
  r.friction_angle = phi;
  return r;
}

}  // namespace

namespace mpm {
void set_last_error(const std::string& msg) { g_last_error = msg; }
}  // namespace mpm

// The engine is shared by everything created from it: mpm_engine_destroy
// drops the caller's reference, and the device stream goes away with the
// last simulation, group or server that still uses it.
struct mpm_engine {
  std::shared_ptr<mpm::Engine> e;
};

struct mpm_sim {
  std::shared_ptr<mpm::Engine> hold;  // first member: released after the group
  mpm::Engine* eng = nullptr;
  std::unique_ptr<mpm::Group> group;
  mpm_config cfg{};
  std::vector<mpm_rheology> rows;  // set_materials rows; empty: cfg.rheology
  std::vector<uint32_t> ids;       // material ids as last set
  std::vector<float> mass, volume; // optional per-particle overrides
  uint32_t sid = 0xffffffffu;
  uint32_t count = 0;
  bool order_prepared = false;
  uint32_t order_capacity = 0;
  bool order_enabled = false;
  bool det_prepared = false;
  bool det_enabled = false;
  bool two_pass = true;  // set_p2g_mode flag (API parity; one scatter serves both)
  uint32_t sort_interval = 0;
  std::vector<float> spheres;  // rigid spheres, 7 floats each (kept across set_particles)
  mpm::DevBuf<float4> render;  // render view positions (max_particles float4), allocated on first use
  uint64_t render_source = 0;  // binding identity of `render`
  uint64_t epoch = 1;
  float dt = 1.0e-4f;
  uint32_t tile_cap = 0;  // new_sparse: grid storage of this many 4^3-node tiles (0: dense)

  std::vector<mpm_rheology> effective_rows() const {
    if (!rows.empty()) return rows;
    return {cfg.rheology};
  }
  void apply_group_settings() {
    const uint32_t interval = order_enabled ? 1u : (sort_interval ? sort_interval : 32u);
    group->sort_interval = interval;
  }
  void invalidate() { ++epoch; }
  // Re-pack the render view after anything that moved particles, on the
  // stream the physics ran on, so a draw queued after it sees this state.
  void refresh_render(cudaStream_t st) {
    if (render.ptr && sid != 0xffffffffu && count) group->pack_positions(sid, render.ptr, st);
  }
};

// All-FP64 simulation (precision studies): FP64 state and grid.
struct mpm_sim64 {
  std::shared_ptr<mpm::Engine> hold;
  mpm::Engine* eng = nullptr;
  mpm_config cfg{};
  mpm::Scene64 sc{};
  uint32_t count = 0;
  mpm::DevBuf<double> pos, vel, C, F, mass, vol, jp, gmass, gmom, gvel, totals;
  mpm::DevBuf<uint32_t> mat, status;

  mpm::State64 state() {
    mpm::State64 st;
    st.n = (int)count;
    st.pos = pos.ptr;
    st.vel = vel.ptr;
    st.C = C.ptr;
    st.F = F.ptr;
    st.mass = mass.ptr;
    st.vol = vol.ptr;
    st.jp = jp.ptr;
    st.mat = mat.ptr;
    st.gmass = gmass.ptr;
    st.gmom = gmom.ptr;
    st.gvel = gvel.ptr;
    st.status = status.ptr;
    return st;
  }
  void set_rows(const mpm_rheology* rows, uint32_t n_rows) {
    sc.n_mat = (int)n_rows;
    for (uint32_t r = 0; r < n_rows; ++r) {
      const mpm_rheology& m = rows[r];
      const double e = m.youngs > 0.f ? (double)m.youngs : (double)cfg.youngs;
      const double nu = m.youngs > 0.f ? (double)m.poisson : (double)cfg.poisson;
      mpm::Mat64& d = sc.mat[r];
      d.rheo = (int)m.kind;
      d.mu = e / (2.0 * (1.0 + nu));
      d.lam = e * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
      d.kappa = (3.0 * d.lam + 2.0 * d.mu) / (2.0 * d.mu);
      d.dp_alpha = m.kind == MPM_RHEOLOGY_SAND ? (double)mpm_dp_alpha(m.friction_angle) : 0.0;
      d.theta_c = m.kind == MPM_RHEOLOGY_SNOW ? (double)m.theta_c : 0.0;
      d.theta_s = m.kind == MPM_RHEOLOGY_SNOW ? (double)m.theta_s : 0.0;
      d.hardening = m.kind == MPM_RHEOLOGY_SNOW ? (double)m.hardening : 0.0;
      d.vdamp = m.kind == MPM_RHEOLOGY_VISCOUS ? (double)m.velocity_damping : 0.0;
      d.adamp = m.kind == MPM_RHEOLOGY_VISCOUS ? (double)m.affine_damping : 0.0;
    }
  }
};

struct mpm_prepared {
  mpm_sim* sim;
  uint64_t epoch;
  float dt;
  uint32_t substeps;
};

struct mpm_batch {
  mpm_sim* sim;
  cudaStream_t stream;
  std::vector<std::pair<float, uint32_t>> work;
  bool done = false;
};

extern "C" {

uint32_t mpm_abi_version(void) { return MOLLA_MPM_ABI_VERSION; }

size_t mpm_last_error(char* buf, size_t size) {
  if (buf && size) {
    const size_t n = std::min(size - 1, g_last_error.size());
    std::memcpy(buf, g_last_error.data(), n);
    buf[n] = 0;
  }
  return g_last_error.size();
}

// ---- engine ----------------------------------------------------------------

int mpm_engine_create(int device, mpm_engine** out) {
  return guard([&] {
    REQUIRE(out, MPM_ERR_INVALID, "null output handle");
    auto* h = new mpm_engine();
    try {
      h->e.reset(new mpm::Engine(device));
    } catch (...) {
      delete h;
      throw;
    }
    *out = h;
  });
}

int mpm_engine_destroy(mpm_engine* engine) {
  return guard([&] { delete engine; });
}

int mpm_engine_check(mpm_engine* engine) {
  return guard([&] {
    REQUIRE(engine, MPM_ERR_INVALID, "null engine");
    engine->e->check();
    cudaError_t e = cudaStreamQuery(engine->e->stream);
    if (e != cudaSuccess && e != cudaErrorNotReady) {
      engine->e->note_error(e);
      mpm::throw_cuda(e, "engine check");
    }
  });
}

int mpm_engine_synchronize(mpm_engine* engine) {
  return guard([&] {
    REQUIRE(engine, MPM_ERR_INVALID, "null engine");
    engine->e->check();
    cudaError_t e = cudaStreamSynchronize(engine->e->stream);
    if (e != cudaSuccess) {
      engine->e->note_error(e);
      mpm::throw_cuda(e, "stream synchronize");
    }
  });
}

uint64_t mpm_engine_launch_count(mpm_engine* engine) { return engine ? engine->e->launches : 0; }

int mpm_selftest_device_wait(mpm_engine* engine, uint32_t* fault_bits, double* waited_ms) {
  return guard([&] {
    REQUIRE(engine && fault_bits, MPM_ERR_INVALID, "null argument");
    mpm::Engine* e = engine->e.get();
    e->check();
    mpm::DevBuf<uint32_t> status(1);
    mpm::DevBuf<unsigned long long> waited(1);
    MPM_CK(cudaMemsetAsync(status.ptr, 0, sizeof(uint32_t), e->stream));
    MPM_CK(cudaMemsetAsync(waited.ptr, 0, sizeof(unsigned long long), e->stream));
    MPM_CK(mpm::launch_selftest_wait(status.ptr, waited.ptr, e->stream));
    e->launches += 1;
    uint32_t bits = 0;
    unsigned long long ns = 0;
    MPM_CK(cudaMemcpyAsync(&bits, status.ptr, sizeof(bits), cudaMemcpyDeviceToHost, e->stream));
    MPM_CK(cudaMemcpyAsync(&ns, waited.ptr, sizeof(ns), cudaMemcpyDeviceToHost, e->stream));
    MPM_CK(cudaStreamSynchronize(e->stream));
    *fault_bits = bits;
    if (waited_ms) *waited_ms = (double)ns * 1.0e-6;
  });
}

void* mpm_engine_stream(mpm_engine* engine) { return engine ? (void*)engine->e->stream : nullptr; }

int mpm_profile_enable(mpm_engine* engine, int enabled) {
  return guard([&] {
    REQUIRE(engine, MPM_ERR_INVALID, "null engine");
    engine->e->profiling = enabled != 0;
  });
}

int mpm_profile_read(mpm_engine* engine, mpm_profile_stage* out, uint32_t cap) {
  return guard([&] {
    REQUIRE(engine && out, MPM_ERR_INVALID, "null argument");
    engine->e->prof_resolve();
    for (uint32_t i = 0; i < cap && i < (uint32_t)mpm::kStages; ++i) {
      out[i].launches = engine->e->prof_count[i];
      out[i].total_ms = engine->e->prof_ms[i];
    }
  });
}

int mpm_profile_reset(mpm_engine* engine) {
  return guard([&] {
    REQUIRE(engine, MPM_ERR_INVALID, "null engine");
    engine->e->prof_resolve();
    for (int i = 0; i < mpm::kStages; ++i) {
      engine->e->prof_ms[i] = 0;
      engine->e->prof_count[i] = 0;
    }
  });
}

// ---- configuration -----------------------------------------------------------

float mpm_dp_alpha(float friction_angle) { return mpm::dp_alpha_of(friction_angle); }

int mpm_config_preset(uint32_t preset, mpm_config* out) {
  return guard([&] {
    REQUIRE(out, MPM_ERR_INVALID, "null config");
    mpm_config c{};
    const float deg30 = 30.0f * 3.14159265358979f / 180.0f;
    c.max_rigid = 8;
    c.cohesion = 0.f;
    c.time_step = MPM_TIME_STEP_EXPLICIT;
    switch (preset) {
      case MPM_PRESET_SAND:  // mpm.rs:540-560
        c.grid_size = 32;
        c.cell_size = 0.05f;
        c.grid_origin[0] = -0.8f, c.grid_origin[1] = 0.f, c.grid_origin[2] = -0.8f;
        c.gravity_y = -9.81f;
        c.youngs = 5.0e3f;
        c.poisson = 0.3f;
        c.friction_angle = deg30;
        c.boundary_friction = 0.5f;
        c.particle_mass = 1.0e-3f;
        c.particle_volume = 1.0e-6f;
        c.max_particles = 16384;
        c.rheology = sand_row(deg30);
        break;
      case MPM_PRESET_SAND_CALIBRATED:  // mpm.rs:585-605 (the implicit step is not built)
        c.grid_size = 48;
        c.cell_size = 0.05f;
        c.grid_origin[0] = -1.2f, c.grid_origin[1] = 0.f, c.grid_origin[2] = -1.2f;
        c.gravity_y = -9.81f;
        c.youngs = 1.0e5f;
        c.poisson = 0.3f;
        c.friction_angle = deg30;
        c.boundary_friction = 0.3f;
        c.particle_mass = 1.5e-3f;
        c.particle_volume = 1.0e-6f;
        c.max_particles = 32768;
        c.rheology = sand_row(deg30);
        c.time_step = MPM_TIME_STEP_IMPLICIT;
        c.jacobi_iters = 3;
        break;
      case MPM_PRESET_SNOW:  // mpm.rs:609-631
        c.grid_size = 32;
        c.cell_size = 0.05f;
        c.grid_origin[0] = -0.8f, c.grid_origin[1] = 0.f, c.grid_origin[2] = -0.8f;
        c.gravity_y = -9.81f;
        c.youngs = 1.4e5f;
        c.poisson = 0.2f;
        c.friction_angle = 0.f;
        c.boundary_friction = 0.5f;
        c.particle_mass = 1.0e-3f;
        c.particle_volume = 1.0e-6f;
        c.max_particles = 16384;
        c.rheology.kind = MPM_RHEOLOGY_SNOW;
        c.rheology.theta_c = 2.5e-2f;
        c.rheology.theta_s = 7.5e-3f;
        c.rheology.hardening = 10.f;
        break;
      case MPM_PRESET_VISCOUS:  // mpm.rs:637-655
        c.grid_size = 32;
        c.cell_size = 0.05f;
        c.grid_origin[0] = -0.8f, c.grid_origin[1] = 0.f, c.grid_origin[2] = -0.8f;
        c.gravity_y = -9.81f;
        c.youngs = 2.0e3f;
        c.poisson = 0.3f;
        c.friction_angle = 0.f;
        c.boundary_friction = 0.8f;
        c.particle_mass = 1.0e-3f;
        c.particle_volume = 1.0e-6f;
        c.max_particles = 16384;
        c.rheology.kind = MPM_RHEOLOGY_VISCOUS;
        c.rheology.velocity_damping = 4.f;
        c.rheology.affine_damping = 8.f;
        break;
      default:
        throw Error(MPM_ERR_INVALID, "unknown MPM preset");
    }
    *out = c;
  });
}

// ---- simulation ---------------------------------------------------------------

static mpm_sim* sim_new(mpm_engine* engine, const mpm_config* cfg, uint32_t tile_cap) {
  REQUIRE(engine && cfg, MPM_ERR_INVALID, "null argument");
  engine->e->check();
  validate_config(*cfg);
  const uint64_t w = (cfg->grid_size + 3u) / 4u;
  REQUIRE(tile_cap <= w * w * w, MPM_ERR_INVALID, "MPM tile pool capacity is invalid");
  REQUIRE(!tile_cap || cfg->time_step != MPM_TIME_STEP_IMPLICIT, MPM_ERR_UNSUPPORTED,
          "sparse MPM grid storage runs the explicit time step only");
  auto* s = new mpm_sim();
  try {
    s->hold = engine->e;
    s->eng = engine->e.get();
    s->cfg = *cfg;
    s->tile_cap = tile_cap;
    const uint64_t cells = tile_cap ? 64ull * tile_cap : (uint64_t)cfg->grid_size * cfg->grid_size * cfg->grid_size;
    s->group.reset(new mpm::Group(s->eng, 1, std::max<uint32_t>(cfg->max_particles, 1), cells));
    s->apply_group_settings();
  } catch (...) {
    delete s;
    throw;
  }
  return s;
}

int mpm_sim_create_sparse(mpm_engine* engine, const mpm_config* cfg, uint32_t tile_capacity, mpm_sim** out) {
  return guard([&] {
    REQUIRE(out, MPM_ERR_INVALID, "null argument");
    REQUIRE(tile_capacity > 0, MPM_ERR_INVALID, "MPM tile pool capacity is invalid");
    *out = sim_new(engine, cfg, tile_capacity);
  });
}

int mpm_sim_create(mpm_engine* engine, const mpm_config* cfg, mpm_sim** out) {
  return guard([&] {
    REQUIRE(engine && cfg && out, MPM_ERR_INVALID, "null argument");
    engine->e->check();
    validate_config(*cfg);
    auto* s = new mpm_sim();
    try {
      s->hold = engine->e;
      s->eng = engine->e.get();
      s->cfg = *cfg;
      const uint64_t n3 = (uint64_t)cfg->grid_size * cfg->grid_size * cfg->grid_size;
      s->group.reset(new mpm::Group(s->eng, 1, std::max<uint32_t>(cfg->max_particles, 1), n3));
      s->apply_group_settings();
    } catch (...) {
      delete s;
      throw;
    }
    *out = s;
  });
}

int mpm_sim_destroy(mpm_sim* sim) {
  return guard([&] { delete sim; });
}

static void sim_reseed(mpm_sim* s, const float* xyz, const float* vel, uint32_t n) {
  if (s->sid != 0xffffffffu) {
    s->group->remove_scene(s->sid);
    s->sid = 0xffffffffu;
  }
  // Material ids persist across reseeds (as the reference's id buffer does):
  // the first n of the last set_materials, zero past its end.
  std::vector<uint32_t> mat;
  const uint32_t* ids = nullptr;
  if (n && s->ids.size() >= n) {
    ids = s->ids.data();
  } else if (n && !s->ids.empty()) {
    mat.assign(n, 0u);
    std::copy(s->ids.begin(), s->ids.end(), mat.begin());
    ids = mat.data();
  }
  const float* mass = s->mass.size() == n && n ? s->mass.data() : nullptr;
  const float* vol = s->volume.size() == n && n ? s->volume.data() : nullptr;
  s->sid = s->group->add_scene(s->cfg, s->effective_rows(), xyz, vel, mass, vol, ids, n, s->dt, s->tile_cap);
  s->count = n;
  s->apply_group_settings();
  if (!s->spheres.empty())
    s->group->set_scene_rigid(s->sid, s->spheres.data(), (uint32_t)(s->spheres.size() / 7), s->eng->stream);
  s->refresh_render(s->eng->stream);
  s->invalidate();
}

int mpm_set_particles(mpm_sim* sim, const float* xyz, const float* vel_or_null, uint32_t n) {
  return guard([&] {
    REQUIRE(sim, MPM_ERR_INVALID, "null simulation");
    REQUIRE(n == 0 || xyz, MPM_ERR_INVALID, "null positions");
    REQUIRE(n <= sim->cfg.max_particles, MPM_ERR_GPU,
            "set_particles: n=" + std::to_string(n) + " > max_particles=" + std::to_string(sim->cfg.max_particles));
    sim->mass.clear();
    sim->volume.clear();
    sim_reseed(sim, xyz, vel_or_null, n);
  });
}

int mpm_set_rigid_spheres(mpm_sim* sim, const float* spheres, uint32_t n) {
  return guard([&] {
    REQUIRE(sim && (spheres || n == 0), MPM_ERR_INVALID, "null argument");
    REQUIRE(n <= sim->cfg.max_rigid, MPM_ERR_GPU,
            "set_rigid_spheres: n=" + std::to_string(n) + " > max_rigid=" + std::to_string(sim->cfg.max_rigid));
    REQUIRE(n <= (uint32_t)mpm::kMaxRigid, MPM_ERR_UNSUPPORTED, "at most 8 rigid spheres per simulation");
    sim->eng->check();
    sim->spheres.assign(spheres, spheres + 7 * (size_t)n);
    if (sim->sid != 0xffffffffu) sim->group->set_scene_rigid(sim->sid, spheres, n, sim->eng->stream);
    sim->invalidate();
  });
}

int mpm_read_rigid_wrenches(mpm_sim* sim, float* out, uint32_t cap, uint32_t* count_out) {
  return guard([&] {
    REQUIRE(sim, MPM_ERR_INVALID, "null simulation");
    sim->eng->check();
    const uint32_t n = (uint32_t)(sim->spheres.size() / 7);
    if (count_out) *count_out = n;
    if (!n) return;
    REQUIRE(out && cap >= n, MPM_ERR_INVALID, "output capacity below the sphere count");
    if (sim->sid == 0xffffffffu) {
      std::fill(out, out + 6 * (size_t)n, 0.f);
      return;
    }
    sim->group->read_scene_wrench(sim->sid, out, n, sim->eng->stream);
  });
}

int mpm_set_particle_mass_volume(mpm_sim* sim, const float* mass_or_null, const float* volume_or_null, uint32_t n) {
  return guard([&] {
    REQUIRE(sim, MPM_ERR_INVALID, "null simulation");
    REQUIRE(n == sim->count, MPM_ERR_INVALID, "mass/volume count must equal the particle count");
    if (!n) return;
    if (mass_or_null) sim->group->write_rows(sim->sid, mpm::MASS, 1, mass_or_null, sim->eng->stream);
    if (volume_or_null) sim->group->write_rows(sim->sid, mpm::VOL, 1, volume_or_null, sim->eng->stream);
    sim->invalidate();
  });
}

int mpm_set_materials(mpm_sim* sim, const mpm_rheology* rows, uint32_t n_rows, const uint32_t* ids, uint32_t n) {
  return guard([&] {
    REQUIRE(sim, MPM_ERR_INVALID, "null simulation");
    REQUIRE(n_rows >= 1 && n_rows <= 8 && rows, MPM_ERR_INVALID,
            "MPM set_materials: 1..=8 material rows required, got " + std::to_string(n_rows));
    REQUIRE(n == sim->count, MPM_ERR_INVALID,
            "MPM set_materials: " + std::to_string(n) + " particle ids for " + std::to_string(sim->count) +
                " particles — seed particles first");
    for (uint32_t i = 0; i < n_rows; ++i) REQUIRE(rows[i].kind <= 2, MPM_ERR_INVALID, "unknown MPM rheology");
    // range check as a branch-free max (vectorises); name the first bad id
    uint32_t top = 0;
    for (uint32_t i = 0; i < n; ++i) top = std::max(top, ids[i]);
    if (top >= n_rows) {
      const uint32_t bad = *std::find_if(ids, ids + n, [&](uint32_t v) { return v >= n_rows; });
      throw Error(MPM_ERR_INVALID, "MPM set_materials: particle material id " + std::to_string(bad) +
                                       " out of range (" + std::to_string(n_rows) + " rows)");
    }
    sim->rows.assign(rows, rows + n_rows);
    sim->ids.assign(ids, ids + n);
    if (sim->sid != 0xffffffffu) {
      sim->group->set_scene_rows(sim->sid, sim->effective_rows());
      sim->group->set_material_ids(sim->sid, ids, n);
    }
    sim->invalidate();
  });
}

int mpm_set_rheology(mpm_sim* sim, const mpm_rheology* rheology) {
  return guard([&] {
    REQUIRE(sim && rheology, MPM_ERR_INVALID, "null argument");
    REQUIRE(rheology->kind <= 2, MPM_ERR_INVALID, "unknown MPM rheology");
    sim->cfg.rheology = *rheology;
    if (rheology->kind == MPM_RHEOLOGY_SAND) sim->cfg.friction_angle = rheology->friction_angle;
    if (sim->sid != 0xffffffffu) {
      sim->group->set_scene_cfg(sim->sid, sim->cfg);
      sim->group->set_scene_rows(sim->sid, sim->effective_rows());
    }
    sim->invalidate();
  });
}

int mpm_set_material(mpm_sim* sim, float youngs, float friction_angle) {
  return guard([&] {
    REQUIRE(sim, MPM_ERR_INVALID, "null simulation");
    sim->cfg.youngs = youngs;
    sim->cfg.friction_angle = friction_angle;
    if (sim->cfg.rheology.kind == MPM_RHEOLOGY_SAND) sim->cfg.rheology.friction_angle = friction_angle;
    if (sim->sid != 0xffffffffu) {
      sim->group->set_scene_cfg(sim->sid, sim->cfg);
      sim->group->set_scene_rows(sim->sid, sim->effective_rows());
    }
    sim->invalidate();
  });
}

int mpm_set_time_step(mpm_sim* sim, uint32_t kind, uint32_t jacobi_iters) {
  return guard([&] {
    REQUIRE(sim, MPM_ERR_INVALID, "null simulation");
    REQUIRE(kind <= MPM_TIME_STEP_IMPLICIT, MPM_ERR_INVALID, "unknown MPM time step");
    sim->cfg.time_step = kind;
    sim->cfg.jacobi_iters = kind == MPM_TIME_STEP_IMPLICIT ? jacobi_iters : 0u;
    if (sim->sid != 0xffffffffu) sim->group->set_scene_cfg(sim->sid, sim->cfg);
    sim->invalidate();
  });
}

int mpm_set_p2g_mode(mpm_sim* sim, int two_pass) {
  return guard([&] {
    REQUIRE(sim, MPM_ERR_INVALID, "null simulation");
    sim->two_pass = two_pass != 0;
    sim->det_enabled = false;
    sim->group->set_deterministic(false);
    sim->invalidate();
  });
}

int mpm_prepare_deterministic_p2g(mpm_sim* sim) {
  return guard([&] {
    REQUIRE(sim, MPM_ERR_INVALID, "null simulation");
    sim->det_prepared = true;
    sim->invalidate();
  });
}

int mpm_set_deterministic_p2g(mpm_sim* sim, int enabled) {
  return guard([&] {
    REQUIRE(sim, MPM_ERR_INVALID, "null simulation");
    if (enabled)
      REQUIRE(sim->det_prepared && sim->order_enabled, MPM_ERR_INVALID,
              "Deterministic P2G requires prepared gather, active or native dense grid, ordering and no deferred "
              "scatter");
    sim->det_enabled = enabled != 0;
    sim->group->set_deterministic(sim->det_enabled);
    sim->invalidate();
  });
}

int mpm_release_deterministic_p2g(mpm_sim* sim) {
  return guard([&] {
    REQUIRE(sim, MPM_ERR_INVALID, "null simulation");
    REQUIRE(!sim->det_enabled, MPM_ERR_INVALID, "Disable deterministic P2G before releasing it");
    if (sim->det_prepared) {
      sim->det_prepared = false;
      sim->invalidate();
    }
  });
}

int mpm_sim_info_get(mpm_sim* sim, mpm_sim_info* out) {
  return guard([&] {
    REQUIRE(sim && out, MPM_ERR_INVALID, "null argument");
    mpm_sim_info i{};
    i.particle_count = sim->count;
    i.uses_two_pass_p2g = sim->two_pass && !sim->det_enabled;
    i.deterministic_p2g = sim->det_enabled;
    i.deterministic_prepared = sim->det_prepared;
    i.tile_ordering = sim->order_enabled;
    i.tile_ordering_capacity = sim->order_prepared ? sim->order_capacity : 0u;
    i.sort_interval = sim->group->sort_interval;
    i.max_particles = sim->cfg.max_particles;
    *out = i;
  });
}

int mpm_sim_config(mpm_sim* sim, mpm_config* out) {
  return guard([&] {
    REQUIRE(sim && out, MPM_ERR_INVALID, "null argument");
    *out = sim->cfg;
  });
}

int mpm_prepare_particle_tile_ordering(mpm_sim* sim, uint32_t capacity) {
  return guard([&] {
    REQUIRE(sim, MPM_ERR_INVALID, "null simulation");
    REQUIRE(capacity != 0 && capacity >= sim->count && capacity <= sim->cfg.max_particles, MPM_ERR_INVALID,
            "MPM particle ordering capacity is invalid");
    if (sim->order_prepared && sim->order_capacity == capacity) return;
    REQUIRE(!sim->det_enabled, MPM_ERR_INVALID, "Disable deterministic P2G before replacing particle ordering");
    sim->order_prepared = true;
    sim->order_capacity = capacity;
    sim->invalidate();
  });
}

int mpm_set_particle_tile_ordering(mpm_sim* sim, int enabled) {
  return guard([&] {
    REQUIRE(sim, MPM_ERR_INVALID, "null simulation");
    REQUIRE(enabled || !sim->det_enabled, MPM_ERR_INVALID, "Disable deterministic P2G before particle ordering");
    REQUIRE(!enabled || (sim->order_prepared && sim->order_capacity >= sim->count), MPM_ERR_INVALID,
            "MPM particle ordering must be prepared for the live count");
    sim->order_enabled = enabled != 0;
    sim->apply_group_settings();
    sim->invalidate();
  });
}

int mpm_set_sort_interval(mpm_sim* sim, uint32_t interval) {
  return guard([&] {
    REQUIRE(sim, MPM_ERR_INVALID, "null simulation");
    sim->sort_interval = interval;
    sim->apply_group_settings();
    // a new interval starts a new cadence: the next call opens with a regrouping
    sim->group->need_regroup = true;
    sim->invalidate();
  });
}

static void sim_check_step(mpm_sim* sim, float dt) {
  REQUIRE(std::isfinite(dt) && dt > 0.f, MPM_ERR_INVALID, "MPM timestep must be finite and positive");
  REQUIRE(!sim->order_enabled || sim->order_capacity >= sim->count, MPM_ERR_INVALID,
          "MPM particle count exceeds prepared ordering capacity");
}

int mpm_step_n(mpm_sim* sim, float dt, uint32_t substeps) {
  return guard([&] {
    REQUIRE(sim, MPM_ERR_INVALID, "null simulation");
    sim->eng->check();
    sim_check_step(sim, dt);
    if (sim->count == 0 || substeps == 0) return;
    sim->dt = dt;
    sim->group->set_scene_dt(sim->sid, dt);
    sim->group->step(substeps, sim->eng->stream);
    sim->refresh_render(sim->eng->stream);
  });
}

int mpm_prepare_step(mpm_sim* sim, float dt, uint32_t substeps, mpm_prepared** out) {
  return guard([&] {
    REQUIRE(sim && out, MPM_ERR_INVALID, "null argument");
    REQUIRE(std::isfinite(dt) && dt > 0.f, MPM_ERR_INVALID, "MPM prepared timestep must be finite and positive");
    sim_check_step(sim, dt);
    *out = new mpm_prepared{sim, sim->epoch, dt, substeps};
  });
}

int mpm_prepared_destroy(mpm_prepared* prepared) {
  return guard([&] { delete prepared; });
}

int mpm_batch_begin(mpm_sim* sim, void* stream, mpm_batch** out) {
  return guard([&] {
    REQUIRE(sim && out, MPM_ERR_INVALID, "null argument");
    *out = new mpm_batch{sim, stream ? (cudaStream_t)stream : sim->eng->stream, {}, false};
  });
}

int mpm_batch_encode_step(mpm_batch* batch, const mpm_prepared* prepared) {
  return guard([&] {
    REQUIRE(batch && prepared, MPM_ERR_INVALID, "null argument");
    REQUIRE(!batch->done, MPM_ERR_INVALID, "MPM command batch already submitted");
    REQUIRE(prepared->sim == batch->sim && prepared->epoch == batch->sim->epoch, MPM_ERR_STALE,
            "MPM prepared step belongs to another simulation or stale configuration");
    if (batch->sim->count == 0 || prepared->substeps == 0) return;
    batch->work.emplace_back(prepared->dt, prepared->substeps);
  });
}

int mpm_batch_submit(mpm_batch* batch) {
  int rc = guard([&] {
    REQUIRE(batch, MPM_ERR_INVALID, "null batch");
    REQUIRE(!batch->done, MPM_ERR_INVALID, "MPM command batch already submitted");
    mpm_sim* sim = batch->sim;
    sim->eng->check();
    cudaStream_t st = batch->stream;
    std::unique_ptr<mpm::OwnedEvent> ev;
    if (st != sim->eng->stream) {
      ev.reset(new mpm::OwnedEvent(cudaEventDisableTiming));
      MPM_CK(cudaEventRecord(*ev, sim->eng->stream));
      MPM_CK(cudaStreamWaitEvent(st, *ev, 0));
    }
    for (const auto& w : batch->work) {
      sim->dt = w.first;
      sim->group->set_scene_dt(sim->sid, w.first);
      sim->group->step_graph(w.second, 1, st);
    }
    if (!batch->work.empty()) sim->refresh_render(st);
    if (ev) {
      MPM_CK(cudaEventRecord(*ev, st));
      MPM_CK(cudaStreamWaitEvent(sim->eng->stream, *ev, 0));
    }
    batch->done = true;
  });
  if (rc == MPM_OK) delete batch;
  return rc;
}

int mpm_batch_cancel(mpm_batch* batch) {
  return guard([&] { delete batch; });
}

int mpm_particle_render_view(mpm_sim* sim, mpm_render_view* out) {
  static std::atomic<uint64_t> next_source{1};
  return guard([&] {
    REQUIRE(sim && out, MPM_ERR_INVALID, "null argument");
    sim->eng->check();
    if (!sim->render.ptr) {
      sim->render.alloc(std::max<uint32_t>(sim->cfg.max_particles, 1));
      sim->render_source = next_source.fetch_add(1);
      sim->refresh_render(sim->eng->stream);
    }
    out->positions = sim->render.ptr;
    out->count = sim->count;
    out->capacity = (uint32_t)sim->render.count;
    out->source = sim->render_source;
    out->live_position_bytes = 16ull * sim->count;
  });
}

int mpm_read_positions(mpm_sim* sim, float* out, uint32_t cap, uint32_t* count_out) {
  return guard([&] {
    REQUIRE(sim, MPM_ERR_INVALID, "null simulation");
    sim->eng->check();
    if (count_out) *count_out = sim->count;
    if (!sim->count || !out || !cap) return;
    if (cap >= sim->count) {
      sim->group->read_rows(sim->sid, mpm::PX, 3, out, sim->eng->stream);
    } else {
      std::vector<float> tmp(3 * (size_t)sim->count);
      sim->group->read_rows(sim->sid, mpm::PX, 3, tmp.data(), sim->eng->stream);
      std::memcpy(out, tmp.data(), 12 * (size_t)cap);
    }
  });
}

int mpm_read_velocities(mpm_sim* sim, float* out, uint32_t cap, uint32_t* count_out) {
  return guard([&] {
    REQUIRE(sim, MPM_ERR_INVALID, "null simulation");
    sim->eng->check();
    if (count_out) *count_out = sim->count;
    if (!sim->count || !out || !cap) return;
    if (cap >= sim->count) {
      sim->group->read_rows(sim->sid, mpm::VX, 3, out, sim->eng->stream);
    } else {
      std::vector<float> tmp(3 * (size_t)sim->count);
      sim->group->read_rows(sim->sid, mpm::VX, 3, tmp.data(), sim->eng->stream);
      std::memcpy(out, tmp.data(), 12 * (size_t)cap);
    }
  });
}

int mpm_read_particle_state(mpm_sim* sim, float* C, float* F, float* jp, uint32_t cap, uint32_t* count_out) {
  return guard([&] {
    REQUIRE(sim, MPM_ERR_INVALID, "null simulation");
    sim->eng->check();
    if (count_out) *count_out = sim->count;
    if (!sim->count) return;
    REQUIRE(cap >= sim->count, MPM_ERR_INVALID, "output capacity below the particle count");
    if (C) sim->group->read_rows(sim->sid, mpm::C0, 9, C, sim->eng->stream);
    if (F) sim->group->read_rows(sim->sid, mpm::F0, 9, F, sim->eng->stream);
    if (jp) sim->group->read_rows(sim->sid, mpm::JP, 1, jp, sim->eng->stream);
  });
}

int mpm_write_particle_state(mpm_sim* sim, const float* C, const float* F, const float* jp, uint32_t n) {
  return guard([&] {
    REQUIRE(sim, MPM_ERR_INVALID, "null simulation");
    sim->eng->check();
    REQUIRE(n == sim->count, MPM_ERR_INVALID, "state count must equal the particle count");
    if (!n) return;
    if (C) sim->group->write_rows(sim->sid, mpm::C0, 9, C, sim->eng->stream);
    if (F) sim->group->write_rows(sim->sid, mpm::F0, 9, F, sim->eng->stream);
    if (jp) sim->group->write_rows(sim->sid, mpm::JP, 1, jp, sim->eng->stream);
  });
}

int mpm_read_grid_mass_momentum(mpm_sim* sim, float* mass, float* momentum, size_t cells) {
  return guard([&] {
    REQUIRE(sim, MPM_ERR_INVALID, "null simulation");
    sim->eng->check();
    const uint64_t n3 = (uint64_t)sim->cfg.grid_size * sim->cfg.grid_size * sim->cfg.grid_size;
    REQUIRE(cells >= n3, MPM_ERR_INVALID, "grid output smaller than grid_size^3");
    if (sim->sid == 0xffffffffu) {
      if (mass) std::memset(mass, 0, n3 * 4);
      if (momentum) std::memset(momentum, 0, n3 * 12);
      return;
    }
    sim->group->read_grid(sim->sid, mass, momentum, sim->eng->stream);
  });
}

int mpm_conservation_totals(mpm_sim* sim, double* out8) {
  return guard([&] {
    REQUIRE(sim && out8, MPM_ERR_INVALID, "null argument");
    sim->eng->check();
    if (sim->sid == 0xffffffffu) {
      for (int i = 0; i < 8; ++i) out8[i] = 0.0;
      return;
    }
    sim->group->totals(sim->sid, out8, sim->eng->stream);
  });
}

int mpm_read_status(mpm_sim* sim, mpm_status_info* out) {
  return guard([&] {
    REQUIRE(sim && out, MPM_ERR_INVALID, "null argument");
    sim->eng->check();
    if (sim->sid == 0xffffffffu) {
      std::memset(out, 0, sizeof(*out));
      return;
    }
    sim->group->status(sim->sid, out, sim->eng->stream);
  });
}

int mpm_reset_fault(mpm_sim* sim) {
  return guard([&] {
    REQUIRE(sim, MPM_ERR_INVALID, "null simulation");
    if (sim->sid != 0xffffffffu) sim->group->reset_status(sim->sid, sim->eng->stream);
  });
}

int mpm_read_sort_permutation(mpm_sim* sim, uint32_t* keys, uint32_t* ids, uint32_t capacity) {
  return guard([&] {
    REQUIRE(sim && keys && ids, MPM_ERR_INVALID, "null argument");
    sim->eng->check();
    REQUIRE(capacity >= sim->count, MPM_ERR_INVALID, "MPM particle ordering capacity is invalid");
    if (sim->sid == 0xffffffffu) {
      for (uint32_t i = 0; i < capacity; ++i) {
        keys[i] = 0xffffffffu;
        ids[i] = i;
      }
      return;
    }
    sim->group->sort_permutation(sim->sid, keys, ids, capacity, sim->eng->stream);
  });
}

static void ensure(mpm::DevBuf<uint32_t>& b, size_t n) {
  if (b.count < n) b.alloc(n);
}

static void engine_sort(mpm::Engine* e, uint32_t* d_keys, uint32_t* d_vals, uint32_t n, uint32_t key_bits,
                        cudaStream_t st) {
  REQUIRE(key_bits >= 1 && key_bits <= 32, MPM_ERR_INVALID, "key_bits must be in 1..=32");
  ensure(e->sk[0], n);
  ensure(e->sk[1], n);
  ensure(e->sv[0], n);
  ensure(e->sv[1], n);
  ensure(e->shist, mpm::sort_hist_words(n));
  uint32_t* ko = nullptr;
  uint32_t* vo = nullptr;
  MPM_CK(mpm::radix_sort_pairs(st, d_keys, d_vals, e->sk[0].ptr, e->sk[1].ptr, e->sv[0].ptr, e->sv[1].ptr,
                               e->shist.ptr, n, (int)key_bits, &ko, &vo, &e->launches));
  MPM_CK(cudaMemcpyAsync(d_keys, ko, (size_t)n * 4, cudaMemcpyDeviceToDevice, st));
  MPM_CK(cudaMemcpyAsync(d_vals, vo, (size_t)n * 4, cudaMemcpyDeviceToDevice, st));
}

int mpm_radix_sort_pairs(mpm_engine* engine, uint32_t* keys, uint32_t* values, uint32_t n, uint32_t key_bits) {
  return guard([&] {
    REQUIRE(engine && (n == 0 || (keys && values)), MPM_ERR_INVALID, "null argument");
    mpm::Engine* e = engine->e.get();
    e->check();
    if (!n) return;
    ensure(e->skin, n);
    ensure(e->svin, n);
    cudaStream_t st = e->stream;
    MPM_CK(cudaMemcpyAsync(e->skin.ptr, keys, (size_t)n * 4, cudaMemcpyHostToDevice, st));
    MPM_CK(cudaMemcpyAsync(e->svin.ptr, values, (size_t)n * 4, cudaMemcpyHostToDevice, st));
    engine_sort(e, e->skin.ptr, e->svin.ptr, n, key_bits, st);
    MPM_CK(cudaMemcpyAsync(keys, e->skin.ptr, (size_t)n * 4, cudaMemcpyDeviceToHost, st));
    MPM_CK(cudaMemcpyAsync(values, e->svin.ptr, (size_t)n * 4, cudaMemcpyDeviceToHost, st));
    cudaError_t err = cudaStreamSynchronize(st);
    if (err != cudaSuccess) {
      e->note_error(err);
      mpm::throw_cuda(err, "radix sort");
    }
  });
}

int mpm_radix_sort_pairs_device(mpm_engine* engine, uint32_t* d_keys, uint32_t* d_values, uint32_t n,
                                uint32_t key_bits, void* stream) {
  return guard([&] {
    REQUIRE(engine && (n == 0 || (d_keys && d_values)), MPM_ERR_INVALID, "null argument");
    mpm::Engine* e = engine->e.get();
    e->check();
    if (!n) return;
    engine_sort(e, d_keys, d_values, n, key_bits, stream ? (cudaStream_t)stream : e->stream);
  });
}

}  // extern "C"

// ---- groups --------------------------------------------------------------------

struct mpm_group {
  std::shared_ptr<mpm::Engine> hold;
  mpm::Engine* eng;
  std::unique_ptr<mpm::Group> g;
};

static std::vector<mpm_rheology> rows_of(const mpm_config& cfg, const mpm_rheology* rows, uint32_t n_rows) {
  if (rows && n_rows) return std::vector<mpm_rheology>(rows, rows + n_rows);
  return {cfg.rheology};
}

extern "C" {

int mpm_group_create(mpm_engine* engine, uint32_t max_scenes, uint64_t max_particles_total, uint64_t max_cells_total,
                     mpm_group** out) {
  return guard([&] {
    REQUIRE(engine && out, MPM_ERR_INVALID, "null argument");
    engine->e->check();
    auto* h = new mpm_group();
    try {
      h->hold = engine->e;
      h->eng = engine->e.get();
      h->g.reset(new mpm::Group(h->eng, max_scenes, max_particles_total, max_cells_total));
    } catch (...) {
      delete h;
      throw;
    }
    *out = h;
  });
}

int mpm_group_destroy(mpm_group* group) {
  return guard([&] { delete group; });
}

int mpm_group_add_scene(mpm_group* group, const mpm_config* cfg, const mpm_rheology* rows, uint32_t n_rows,
                        const float* xyz, const uint32_t* ids_or_null, uint32_t n, float dt, uint32_t* scene_id) {
  return guard([&] {
    REQUIRE(group && cfg && scene_id, MPM_ERR_INVALID, "null argument");
    REQUIRE(n == 0 || xyz, MPM_ERR_INVALID, "null positions");
    validate_config(*cfg);
    REQUIRE(std::isfinite(dt) && dt > 0.f, MPM_ERR_INVALID, "MPM timestep must be finite and positive");
    auto r = rows_of(*cfg, rows, n_rows);
    REQUIRE(r.size() <= 8, MPM_ERR_INVALID, "MPM scene needs 1..=8 material rows");
    if (ids_or_null)
      for (uint32_t i = 0; i < n; ++i)
        REQUIRE(ids_or_null[i] < r.size(), MPM_ERR_INVALID, "particle material id out of range");
    *scene_id = group->g->add_scene(*cfg, r, xyz, nullptr, nullptr, nullptr, ids_or_null, n, dt);
  });
}

int mpm_group_add_scene_sparse(mpm_group* group, const mpm_config* cfg, const mpm_rheology* rows, uint32_t n_rows,
                               const float* xyz, const uint32_t* ids_or_null, uint32_t n, float dt,
                               uint32_t tile_capacity, uint32_t* scene_id) {
  return guard([&] {
    REQUIRE(group && cfg && scene_id, MPM_ERR_INVALID, "null argument");
    REQUIRE(n == 0 || xyz, MPM_ERR_INVALID, "null positions");
    REQUIRE(tile_capacity > 0, MPM_ERR_INVALID, "MPM tile pool capacity is invalid");
    validate_config(*cfg);
    REQUIRE(std::isfinite(dt) && dt > 0.f, MPM_ERR_INVALID, "MPM timestep must be finite and positive");
    auto r = rows_of(*cfg, rows, n_rows);
    REQUIRE(r.size() <= 8, MPM_ERR_INVALID, "MPM scene needs 1..=8 material rows");
    if (ids_or_null)
      for (uint32_t i = 0; i < n; ++i)
        REQUIRE(ids_or_null[i] < r.size(), MPM_ERR_INVALID, "particle material id out of range");
    *scene_id = group->g->add_scene(*cfg, r, xyz, nullptr, nullptr, nullptr, ids_or_null, n, dt, tile_capacity);
  });
}

int mpm_group_remove_scene(mpm_group* group, uint32_t scene_id) {
  return guard([&] {
    REQUIRE(group, MPM_ERR_INVALID, "null group");
    group->g->remove_scene(scene_id);
  });
}

int mpm_group_step(mpm_group* group, uint32_t substeps) {
  return guard([&] {
    REQUIRE(group, MPM_ERR_INVALID, "null group");
    group->g->step(substeps, group->eng->stream);
  });
}

int mpm_group_step_graph(mpm_group* group, uint32_t substeps, uint32_t repeat) {
  return guard([&] {
    REQUIRE(group, MPM_ERR_INVALID, "null group");
    group->g->step_graph(substeps, repeat, group->eng->stream);
  });
}

int mpm_group_read_positions(mpm_group* group, uint32_t scene_id, float* out, uint32_t cap, uint32_t* count_out) {
  return guard([&] {
    REQUIRE(group, MPM_ERR_INVALID, "null group");
    REQUIRE(scene_id < group->g->scenes.size() && group->g->scenes[scene_id].live, MPM_ERR_INVALID,
            "unknown MPM scene");
    const uint32_t n = group->g->scenes[scene_id].n;
    if (count_out) *count_out = n;
    if (!out || !n) return;
    REQUIRE(cap >= n, MPM_ERR_INVALID, "output capacity below the particle count");
    group->g->read_rows(scene_id, mpm::PX, 3, out, group->eng->stream);
  });
}

int mpm_group_read_status(mpm_group* group, uint32_t scene_id, mpm_status_info* out) {
  return guard([&] {
    REQUIRE(group && out, MPM_ERR_INVALID, "null argument");
    REQUIRE(scene_id < group->g->scenes.size() && group->g->scenes[scene_id].live, MPM_ERR_INVALID,
            "unknown MPM scene");
    group->g->status(scene_id, out, group->eng->stream);
  });
}

static const uint32_t kDefaultCands[] = {4, 8, 16, 32, 64, 128};

int mpm_group_autotune(mpm_group* group, uint32_t probe_substeps, const uint32_t* candidates, uint32_t n_candidates,
                       float* ms_per_substep, uint32_t* chosen) {
  return guard([&] {
    REQUIRE(group, MPM_ERR_INVALID, "null group");
    const uint32_t* c = candidates ? candidates : kDefaultCands;
    const uint32_t nc = candidates ? n_candidates : 6;
    REQUIRE(nc >= 1 && nc <= 64, MPM_ERR_INVALID, "1..=64 candidates required");
    for (uint32_t i = 0; i < nc; ++i) REQUIRE(c[i] >= 1, MPM_ERR_INVALID, "intervals must be >= 1");
    const uint32_t best = group->g->autotune(probe_substeps, c, (int)nc, ms_per_substep, group->eng->stream);
    if (chosen) *chosen = best;
  });
}

int mpm_autotune(mpm_sim* sim, float dt, uint32_t probe_substeps, const uint32_t* candidates, uint32_t n_candidates,
                 float* ms_per_substep, uint32_t* chosen) {
  return guard([&] {
    REQUIRE(sim, MPM_ERR_INVALID, "null simulation");
    sim_check_step(sim, dt);
    REQUIRE(!sim->order_enabled, MPM_ERR_INVALID, "particle ordering fixes the interval at one substep");
    const uint32_t* c = candidates ? candidates : kDefaultCands;
    const uint32_t nc = candidates ? n_candidates : 6;
    REQUIRE(nc >= 1 && nc <= 64, MPM_ERR_INVALID, "1..=64 candidates required");
    for (uint32_t i = 0; i < nc; ++i) REQUIRE(c[i] >= 1, MPM_ERR_INVALID, "intervals must be >= 1");
    if (sim->count == 0) {
      if (chosen) *chosen = sim->group->sort_interval;
      return;
    }
    sim->group->set_scene_dt(sim->sid, dt);
    const uint32_t best = sim->group->autotune(probe_substeps, c, (int)nc, ms_per_substep, sim->eng->stream);
    sim->sort_interval = best;
    sim->apply_group_settings();
    if (chosen) *chosen = best;
  });
}

static void shapes_to_c(const mpm::Group::Shapes& sh, mpm_shapes* out) {
  std::memset(out, 0, sizeof(*out));
  out->sort_interval = sh.interval;
  out->item_particles = sh.item_particles;
  out->fused = sh.fused;
  out->gather_ctas_per_sm = sh.gather_per_sm;
  out->scatter_ctas_per_sm = sh.scatter_per_sm;
}

static void tune_shapes(mpm::Group& g, uint32_t probe_substeps, mpm_shapes* chosen, mpm_tune_probe* probes,
                        uint32_t cap, uint32_t* n_probes, cudaStream_t st) {
  using G = mpm::Group;
  std::vector<G::Probe> out;
  const G::Shapes sh = g.autotune_shapes(
      probe_substeps ? probe_substeps : 32,
      {{G::kKnobInterval, {}}, {G::kKnobItem, {}}, {G::kKnobFused, {}}, {G::kKnobGatherCtas, {}},
       {G::kKnobScatterCtas, {}}},
      &out, st);
  if (chosen) shapes_to_c(sh, chosen);
  if (probes)
    for (uint32_t i = 0; i < cap && i < out.size(); ++i) probes[i] = {out[i].knob, out[i].value, out[i].ms};
  if (n_probes) *n_probes = (uint32_t)out.size();
}

int mpm_group_autotune_shapes(mpm_group* group, uint32_t probe_substeps, mpm_shapes* chosen, mpm_tune_probe* probes,
                              uint32_t cap, uint32_t* n_probes) {
  return guard([&] {
    REQUIRE(group, MPM_ERR_INVALID, "null group");
    tune_shapes(*group->g, probe_substeps, chosen, probes, cap, n_probes, group->eng->stream);
  });
}

int mpm_autotune_shapes(mpm_sim* sim, float dt, uint32_t probe_substeps, mpm_shapes* chosen, mpm_tune_probe* probes,
                        uint32_t cap, uint32_t* n_probes) {
  return guard([&] {
    REQUIRE(sim, MPM_ERR_INVALID, "null simulation");
    sim_check_step(sim, dt);
    REQUIRE(!sim->order_enabled, MPM_ERR_INVALID, "particle ordering fixes the interval at one substep");
    if (sim->count == 0) {
      if (chosen) shapes_to_c(sim->group->shapes(), chosen);
      if (n_probes) *n_probes = 0;
      return;
    }
    sim->group->set_scene_dt(sim->sid, dt);
    tune_shapes(*sim->group, probe_substeps, chosen, probes, cap, n_probes, sim->eng->stream);
    sim->sort_interval = sim->group->sort_interval;
    sim->apply_group_settings();
    sim->invalidate();
  });
}

int mpm_group_get_shapes(mpm_group* group, mpm_shapes* out) {
  return guard([&] {
    REQUIRE(group && out, MPM_ERR_INVALID, "null argument");
    shapes_to_c(group->g->shapes(), out);
  });
}

int mpm_group_set_shapes(mpm_group* group, const mpm_shapes* in) {
  return guard([&] {
    REQUIRE(group && in, MPM_ERR_INVALID, "null argument");
    REQUIRE(in->sort_interval >= 1, MPM_ERR_INVALID, "the regroup interval must be at least 1");
    mpm::Group::Shapes sh{in->sort_interval, in->item_particles, in->fused ? 1u : 0u, in->gather_ctas_per_sm,
                          in->scatter_ctas_per_sm};
    group->g->apply_shapes(sh);
  });
}

int mpm_group_set_deterministic(mpm_group* group, int enabled) {
  return guard([&] {
    REQUIRE(group, MPM_ERR_INVALID, "null group");
    group->g->set_deterministic(enabled != 0);
  });
}

int mpm_group_scene_count(mpm_group* group, uint32_t* count) {
  return guard([&] {
    REQUIRE(group && count, MPM_ERR_INVALID, "null argument");
    *count = group->g->live_scenes();
  });
}

int mpm_group_tune(mpm_group* group, uint32_t chunk, uint32_t sort_interval) {
  return guard([&] {
    REQUIRE(group, MPM_ERR_INVALID, "null group");
    (void)chunk;  // work items are whole 4^3 tiles
    group->g->sort_interval = sort_interval ? sort_interval : 32;
  });
}

}  // extern "C"

// ---- serving -----------------------------------------------------------------------

namespace {
struct Ticket {
  uint64_t id = 0;
  mpm_config cfg{};
  std::vector<mpm_rheology> rows;
  std::vector<float> xyz;
  std::vector<uint32_t> ids;
  uint32_t n = 0;
  float dt = 0.f;
  uint32_t steps = 0, remaining = 0;
  uint32_t state = 0;  // 0 queued, 1 running, 2 done, 3 faulted
  uint32_t sid = 0xffffffffu;
  uint32_t counted = 0;  // substeps launched for it (counted into particle_steps)
  mpm_status_info status{};  // device status word at retirement
  uint64_t bytes = 0;
  uint32_t tile_cap = 0;  // sparse grid storage when it saves memory (0: dense)
  std::vector<float> result;
  double t_submit = 0, t_admit = 0;
};

// Tile capacity for a served scene: the 4^3-node tiles of the particles'
// stencil bounding box, widened by 2 tiles (8 cells) on every side for the
// motion of the scene's lifetime and clamped to the grid; 0 (dense storage)
// when that is more than half the grid's tiles.  A scene that spreads beyond
// it latches the tile-overflow bit and stops.
uint32_t served_tile_capacity(const mpm_config& cfg, const float* xyz, uint32_t n) {
  const uint32_t w = (cfg.grid_size + 3u) / 4u;
  const uint64_t all = (uint64_t)w * w * w;
  if (n == 0) return 0;
  int lo[3] = {INT32_MAX, INT32_MAX, INT32_MAX}, hi[3] = {INT32_MIN, INT32_MIN, INT32_MIN};
  const float inv_dx = 1.0f / cfg.cell_size;
  for (uint32_t i = 0; i < n; ++i)
    for (int a = 0; a < 3; ++a) {
      const float xp = (xyz[3 * (size_t)i + a] - cfg.grid_origin[a]) * inv_dx;
      if (!std::isfinite(xp)) return 0;
      const int b = (int)std::floor(xp - 0.5f) - cfg.grid_window_cells[a];
      lo[a] = std::min(lo[a], b);
      hi[a] = std::max(hi[a], b + 2);
    }
  uint64_t tiles = 1;
  for (int a = 0; a < 3; ++a) {
    const int t0 = std::max(0, (std::max(lo[a], 0) >> 2) - 2);
    const int t1 = std::min((int)w - 1, (std::min(hi[a], (int)cfg.grid_size - 1) >> 2) + 2);
    tiles *= (uint64_t)std::max(t1 - t0 + 1, 1);
  }
  return 2 * tiles <= all ? (uint32_t)tiles : 0u;
}
double now_ms() {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
double pct(std::vector<double> v, double q) {
  if (v.empty()) return 0.0;
  std::sort(v.begin(), v.end());
  const double pos = q * (double)(v.size() - 1);
  const size_t i = (size_t)pos;
  const double f = pos - (double)i;
  return i + 1 < v.size() ? v[i] * (1 - f) + v[i + 1] * f : v[i];
}
}  // namespace

// Device bytes a resident particle occupies in a group pool.
constexpr uint64_t kServerBytesPerParticle = 2ull * mpm::kPlanes * 4ull + 64ull + 44ull;

struct mpm_server {
  std::shared_ptr<mpm::Engine> hold;
  mpm::Engine* eng;
  std::unique_ptr<mpm::Group> g;
  uint64_t budget = 0;
  uint64_t resident = 0;
  std::deque<uint64_t> queue;
  std::map<uint64_t, Ticket> tickets;
  uint64_t next_id = 1;
  uint64_t admitted = 0, completed = 0, faulted = 0, particle_steps = 0;
  std::vector<uint32_t> status_w;  // status words read at each tick's completion
  std::vector<double> tick_ms, queue_ms;
  double admit_ms = 0, step_ms = 0, retire_ms = 0;
  uint64_t ticks = 0;
  bool in_flight = false;  // a tick launched and not yet completed
  uint32_t in_flight_len = 0;
  ~mpm_server() {
    if (in_flight && eng) cudaEventSynchronize(*e1);
  }
  std::unique_ptr<mpm::OwnedEvent> e0, e1;  // tick timing
};

extern "C" {

int mpm_server_create(mpm_engine* engine, uint64_t hbm_budget_bytes, uint32_t max_scenes, mpm_server** out) {
  return guard([&] {
    REQUIRE(engine && out && hbm_budget_bytes > 0, MPM_ERR_INVALID, "invalid argument");
    engine->e->check();
    auto* s = new mpm_server();
    try {
      s->hold = engine->e;
      s->eng = engine->e.get();
      s->budget = hbm_budget_bytes;
      // Split the budget: particle pool 60% (two 27-plane buffers, the
      // 64-byte scatter record and eleven index/key words per slot), grid
      // pool 40% (three float4 arrays per cell).
      const uint64_t per_particle = kServerBytesPerParticle;
      const uint64_t particles = std::min<uint64_t>(hbm_budget_bytes / 5 * 3 / per_particle, 0x7fff0000ull);
      const uint64_t cells = hbm_budget_bytes / 5 * 2 / 48ull;
      s->g.reset(new mpm::Group(s->eng, std::max<uint32_t>(max_scenes, 1), particles, cells));
      s->e0.reset(new mpm::OwnedEvent());
      s->e1.reset(new mpm::OwnedEvent());
    } catch (...) {
      delete s;
      throw;
    }
    *out = s;
  });
}

int mpm_server_destroy(mpm_server* server) {
  return guard([&] {
    if (!server) return;
    delete server;
  });
}

int mpm_server_submit(mpm_server* server, const mpm_config* cfg, const mpm_rheology* rows, uint32_t n_rows,
                      const float* xyz, const uint32_t* ids_or_null, uint32_t n, float dt, uint32_t steps,
                      uint64_t* ticket) {
  return guard([&] {
    REQUIRE(server && cfg && ticket && (n == 0 || xyz), MPM_ERR_INVALID, "null argument");
    validate_config(*cfg);
    REQUIRE(std::isfinite(dt) && dt > 0.f, MPM_ERR_INVALID, "MPM timestep must be finite and positive");
    Ticket t;
    t.id = server->next_id++;
    t.cfg = *cfg;
    t.rows = rows_of(*cfg, rows, n_rows);
    t.xyz.assign(xyz, xyz + 3 * (size_t)n);
    if (ids_or_null) t.ids.assign(ids_or_null, ids_or_null + n);
    t.n = n;
    t.dt = dt;
    t.steps = t.remaining = steps;
    // sparse grid storage when the particles occupy a small part of the grid
    // and the configuration allows it (explicit time step)
    t.tile_cap = cfg->time_step == MPM_TIME_STEP_IMPLICIT ? 0u : served_tile_capacity(*cfg, xyz, n);
    const uint64_t wt = (cfg->grid_size + 3u) / 4u;
    const uint64_t n3 = t.tile_cap ? 64ull * t.tile_cap : (uint64_t)cfg->grid_size * cfg->grid_size * cfg->grid_size;
    // particles, grid nodes (two accumulators and the velocity), and with
    // sparse storage the per-tile map and marks
    t.bytes = (uint64_t)n * kServerBytesPerParticle + (n3 + 255) / 256 * 256 * 48ull + (t.tile_cap ? wt * wt * wt * 5 : 0);
    REQUIRE(n <= server->g->cap && (n3 + 255) / 256 * 256 <= server->g->cell_cap && t.bytes <= server->budget,
            MPM_ERR_INVALID, "scene exceeds the server's HBM budget or pools");
    t.t_submit = now_ms();
    *ticket = t.id;
    server->queue.push_back(t.id);
    server->tickets.emplace(t.id, std::move(t));
  });
}

// Completes the tick in flight: waits for it, records its time, and retires
// the scenes that finished in it (their results are read, their slots go
// back at the next regrouping).
static void server_complete_tick(mpm_server* server) {
  if (!server->in_flight) return;
  mpm::Group& g = *server->g;
  cudaStream_t st = server->eng->stream;
  const double t0 = now_ms();
  MPM_CK(cudaEventSynchronize(*server->e1));
  server->in_flight = false;
  float ms = 0.f;
  MPM_CK(cudaEventElapsedTime(&ms, *server->e0, *server->e1));
  const uint32_t len = server->in_flight_len;
  server->tick_ms.push_back(ms / (float)len);
  const double t_ret0 = now_ms();
  server->step_ms += t_ret0 - t0;
  // One copy of every scene's status word: a scene whose fault latch is set
  // (a non-finite state, a sparse grid out of tiles) stands frozen on the
  // device, so it is retired now as faulted instead of running out its
  // budget, and the substeps it did not take leave the step count.
  g.status_words(server->status_w, st);
  for (auto& kv : server->tickets) {
    Ticket& t = kv.second;
    if (t.state != 1) continue;
    const uint32_t* w = server->status_w.data() + (size_t)t.sid * mpm::kStatusWords;
    const bool fault = w[0] != 0u;
    t.remaining = fault ? 0 : (t.remaining > len ? t.remaining - len : 0);
    if (t.remaining == 0) {
      t.status.fault_bits = w[0];
      t.status.numerical_fault = (w[0] & mpm::kFaultNumerical) ? 1u : 0u;
      t.status.completed_substeps = (w[2] != 0u && w[1] > w[2]) ? w[2] : w[1];
      t.result.resize(3 * (size_t)t.n);
      if (t.n) g.read_rows(t.sid, mpm::PX, 3, t.result.data(), st);
      g.retire_scene(t.sid);
      server->resident -= t.bytes;
      if (fault) {
        if (t.counted > t.status.completed_substeps)
          server->particle_steps -= (uint64_t)t.n * (t.counted - t.status.completed_substeps);
        t.state = 3;
        server->faulted++;
      } else {
        t.state = 2;
        server->completed++;
      }
    }
  }
  server->retire_ms += now_ms() - t_ret0;
}

int mpm_server_run(mpm_server* server, uint32_t ticks, uint32_t substeps_per_tick) {
  return guard([&] {
    REQUIRE(server && substeps_per_tick > 0, MPM_ERR_INVALID, "invalid argument");
    mpm::Group& g = *server->g;
    cudaStream_t st = server->eng->stream;
    for (uint32_t tick = 0; tick < ticks; ++tick) {
      server_complete_tick(server);
      const double t_admit0 = now_ms();
      // admit in arrival order while the budget and pools allow
      while (!server->queue.empty()) {
        Ticket& t = server->tickets.at(server->queue.front());
        if (t.steps == 0) {
          // nothing to step: the result is the submitted state
          t.result = t.xyz;
          t.state = 2;
          t.t_admit = now_ms();
          server->queue_ms.push_back(t.t_admit - t.t_submit);
          server->admitted++;
          server->completed++;
          server->queue.pop_front();
          continue;
        }
        if (server->resident + t.bytes > server->budget) break;
        uint32_t sid = 0;
        bool added = false;
        for (int attempt = 0; attempt < 2 && !added; ++attempt) {
          try {
            sid = g.add_scene(t.cfg, t.rows, t.xyz.data(), nullptr, nullptr, nullptr,
                              t.ids.empty() ? nullptr : t.ids.data(), t.n, t.dt, t.tile_cap);
            added = true;
          } catch (const Error& e) {
            if (e.code != MPM_ERR_BUSY) throw;
            // the pools may be held by retired scenes awaiting compaction
            if (attempt == 0 && g.n_retiring) g.compact(st);
            else break;
          }
        }
        if (!added) break;
        // the scene stops on the device after exactly its requested substeps
        g.set_scene_budget(sid, t.steps, st, /*fresh=*/true);
        t.sid = sid;
        t.state = 1;
        t.t_admit = now_ms();
        server->queue_ms.push_back(t.t_admit - t.t_submit);
        server->resident += t.bytes;
        server->admitted++;
        server->queue.pop_front();
        std::vector<float>().swap(t.xyz);
      }
      // One tick of a fixed length through a captured graph: every resident
      // scene advances min(remaining, substeps_per_tick) substeps (a scene
      // whose budget ends inside the tick stands still for the rest of it).
      const double t_step0 = now_ms();
      server->admit_ms += t_step0 - t_admit0;
      const uint32_t len = substeps_per_tick;
      uint64_t parts = 0;
      for (auto& kv : server->tickets)
        if (kv.second.state == 1) {
          const uint32_t k = std::min(kv.second.remaining, len);
          parts += (uint64_t)kv.second.n * k;
          kv.second.counted += k;
        }
      if (parts == 0 && g.live_scenes() == 0) {
        if (server->queue.empty()) break;
        continue;
      }
      // the tick's events bracket its graph launch alone: a capture or
      // update of the graph before it is host time (graph_build_ms)
      g.step_graph(len, 1, st, *server->e0, *server->e1);
      // The tick runs on the GPU while the caller goes on (submitting
      // requests); the next run, poll or stats call completes it.
      server->in_flight = true;
      server->in_flight_len = len;
      server->particle_steps += parts;
      server->ticks++;
      server->step_ms += now_ms() - t_step0;
    }
  });
}

int mpm_server_poll(mpm_server* server, uint64_t ticket, uint32_t* state, float* positions_out, uint32_t cap,
                    uint32_t* count_out) {
  return guard([&] {
    REQUIRE(server && state, MPM_ERR_INVALID, "null argument");
    server_complete_tick(server);
    auto it = server->tickets.find(ticket);
    REQUIRE(it != server->tickets.end(), MPM_ERR_INVALID, "unknown ticket");
    Ticket& t = it->second;
    *state = t.state;
    if (count_out) *count_out = t.n;
    if ((t.state == 2 || t.state == 3) && positions_out) {
      REQUIRE(cap >= t.n, MPM_ERR_INVALID, "output capacity below the particle count");
      std::memcpy(positions_out, t.result.data(), 12 * (size_t)t.n);
    }
  });
}

int mpm_server_ticket_status(mpm_server* server, uint64_t ticket, mpm_status_info* out) {
  return guard([&] {
    REQUIRE(server && out, MPM_ERR_INVALID, "null argument");
    server_complete_tick(server);
    auto it = server->tickets.find(ticket);
    REQUIRE(it != server->tickets.end(), MPM_ERR_INVALID, "unknown ticket");
    const Ticket& t = it->second;
    REQUIRE(t.state >= 2, MPM_ERR_INVALID, "the request has not finished");
    *out = t.status;
  });
}

int mpm_blake3(const void* data, size_t len, uint8_t* out32) {
  return guard([&] {
    REQUIRE((data || len == 0) && out32, MPM_ERR_INVALID, "null argument");
    mpm::Blake3 h;
    h.update(static_cast<const uint8_t*>(data), len);
    h.finalize(out32);
  });
}

int mpm_checkpoint_reencode(const uint8_t* bytes, size_t len, uint32_t max_particles, uint8_t* out, size_t cap,
                            size_t* size_out, uint32_t* count_out) {
  return guard([&] {
    REQUIRE(bytes || len == 0, MPM_ERR_INVALID, "null argument");
    const mpm::SoilCheckpoint k = mpm::decode_checkpoint(bytes, len, max_particles);
    if (count_out) *count_out = k.count;
    if (!out) {
      if (size_out) *size_out = mpm::checkpoint_bytes(k.window[0] || k.window[1] || k.window[2],
                                                      (uint32_t)k.materials.size(), k.count);
      return;
    }
    const std::vector<uint8_t> enc = mpm::encode_checkpoint(k);
    if (size_out) *size_out = enc.size();
    REQUIRE(cap >= enc.size(), MPM_ERR_INVALID, "checkpoint buffer too small");
    std::memcpy(out, enc.data(), enc.size());
  });
}

int mpm_checkpoint_save(mpm_sim* sim, uint8_t* out, size_t cap, size_t* size_out) {
  return guard([&] {
    REQUIRE(sim && size_out, MPM_ERR_INVALID, "null argument");
    sim->eng->check();
    const mpm_config& c = sim->cfg;
    const bool lattice = c.grid_window_cells[0] || c.grid_window_cells[1] || c.grid_window_cells[2];
    const size_t need = mpm::checkpoint_bytes(lattice, (uint32_t)sim->rows.size(), sim->count);
    *size_out = need;
    if (!out) return;
    REQUIRE(cap >= need, MPM_ERR_INVALID, "checkpoint buffer too small");
    bool ext = c.rheology.youngs != 0.f || c.rheology.poisson != 0.f;
    for (const mpm_rheology& r : sim->rows) ext = ext || r.youngs != 0.f || r.poisson != 0.f;
    REQUIRE(!ext, MPM_ERR_UNSUPPORTED,
            "MPM soil checkpoint: the format holds one Young's modulus and Poisson ratio; per-material values "
            "cannot be archived");
    if (sim->group && sim->sid != 0xffffffffu) {
      mpm_status_info st{};
      sim->group->status(sim->sid, &st, sim->eng->stream);
      REQUIRE(st.fault_bits == 0, MPM_ERR_FAULT,
              "MPM soil checkpoint: latched grid fault; incomplete state cannot be archived");
    }
    mpm::SoilCheckpoint k;
    k.cfg = c;
    for (int a = 0; a < 3; ++a) k.window[a] = c.grid_window_cells[a];
    k.materials = sim->rows;
    k.count = sim->count;
    const size_t n = sim->count;
    k.words.assign(n * mpm::kCheckpointWordsPerParticle, 0u);
    if (n) {
      std::vector<float> x(3 * n), v(3 * n), C(9 * n), F(9 * n), vol(n), mass(n), jp(n);
      cudaStream_t s = sim->eng->stream;
      sim->group->read_rows(sim->sid, mpm::PX, 3, x.data(), s);
      sim->group->read_rows(sim->sid, mpm::VX, 3, v.data(), s);
      sim->group->read_rows(sim->sid, mpm::C0, 9, C.data(), s);
      sim->group->read_rows(sim->sid, mpm::F0, 9, F.data(), s);
      sim->group->read_rows(sim->sid, mpm::VOL, 1, vol.data(), s);
      sim->group->read_rows(sim->sid, mpm::MASS, 1, mass.data(), s);
      sim->group->read_rows(sim->sid, mpm::JP, 1, jp.data(), s);
      auto bits = [](float f) {
        uint32_t u;
        std::memcpy(&u, &f, 4);
        return u;
      };
      uint32_t* w = k.words.data();
      for (size_t i = 0; i < n; ++i)
        for (int a = 0; a < 3; ++a) w[4 * i + a] = bits(x[3 * i + a]);
      w += 4 * n;
      for (size_t i = 0; i < n; ++i)
        for (int a = 0; a < 3; ++a) w[4 * i + a] = bits(v[3 * i + a]);
      w += 4 * n;
      for (size_t i = 0; i < n; ++i)
        for (int col = 0; col < 3; ++col)
          for (int r = 0; r < 3; ++r) w[12 * i + 4 * col + r] = bits(C[9 * i + 3 * col + r]);
      w += 12 * n;
      for (size_t i = 0; i < n; ++i)
        for (int col = 0; col < 3; ++col)
          for (int r = 0; r < 3; ++r) w[12 * i + 4 * col + r] = bits(F[9 * i + 3 * col + r]);
      w += 12 * n;
      for (size_t i = 0; i < n; ++i) w[i] = bits(vol[i]);
      w += n;
      for (size_t i = 0; i < n; ++i) w[i] = bits(mass[i]);
      w += n;
      for (size_t i = 0; i < n; ++i) w[i] = bits(jp[i]);
      w += n;
      for (size_t i = 0; i < n; ++i) w[i] = sim->ids.size() == n ? sim->ids[i] : 0u;
      // tire compaction (4 words per particle): no tire coupling here, zeros
    }
    mpm::validate_checkpoint(k);
    const std::vector<uint8_t> enc = mpm::encode_checkpoint(k);
    std::memcpy(out, enc.data(), enc.size());
    *size_out = enc.size();
  });
}

namespace {
void must(int rc) {
  if (rc != MPM_OK) throw mpm::Error(rc, g_last_error);
}
}  // namespace

int mpm_checkpoint_load(mpm_sim* sim, const uint8_t* bytes, size_t len) {
  return guard([&] {
    REQUIRE(sim && (bytes || len == 0), MPM_ERR_INVALID, "null argument");
    sim->eng->check();
    const mpm::SoilCheckpoint k = mpm::decode_checkpoint(bytes, len, sim->cfg.max_particles);
    REQUIRE(sim->spheres.empty(), MPM_ERR_INVALID,
            "MPM soil checkpoint: incompatible configuration, capacity or attached rigid bodies");
    const int32_t* w0 = sim->cfg.grid_window_cells;
    REQUIRE(mpm::checkpoint_config_compatible(k.cfg, sim->cfg) && k.window[0] == w0[0] && k.window[1] == w0[1] &&
                k.window[2] == w0[2] && k.count <= sim->cfg.max_particles,
            MPM_ERR_INVALID, "MPM soil checkpoint: incompatible configuration or capacity");
    const size_t n = k.count;
    std::vector<float> x(3 * n), v(3 * n), C(9 * n), F(9 * n), vol(n), mass(n), jp(n);
    std::vector<uint32_t> ids(n);
    auto flt = [](uint32_t u) {
      float f;
      std::memcpy(&f, &u, 4);
      return f;
    };
    const uint32_t* w = k.words.data();
    for (size_t i = 0; i < n; ++i)
      for (int a = 0; a < 3; ++a) x[3 * i + a] = flt(w[4 * i + a]);
    w += 4 * n;
    for (size_t i = 0; i < n; ++i)
      for (int a = 0; a < 3; ++a) v[3 * i + a] = flt(w[4 * i + a]);
    w += 4 * n;
    for (size_t i = 0; i < n; ++i)
      for (int col = 0; col < 3; ++col)
        for (int r = 0; r < 3; ++r) C[9 * i + 3 * col + r] = flt(w[12 * i + 4 * col + r]);
    w += 12 * n;
    for (size_t i = 0; i < n; ++i)
      for (int col = 0; col < 3; ++col)
        for (int r = 0; r < 3; ++r) F[9 * i + 3 * col + r] = flt(w[12 * i + 4 * col + r]);
    w += 12 * n;
    for (size_t i = 0; i < n; ++i) vol[i] = flt(w[i]);
    w += n;
    for (size_t i = 0; i < n; ++i) mass[i] = flt(w[i]);
    w += n;
    for (size_t i = 0; i < n; ++i) jp[i] = flt(w[i]);
    w += n;
    for (size_t i = 0; i < n; ++i) ids[i] = w[i];
    const uint32_t un = (uint32_t)n;
    must(mpm_set_particles(sim, n ? x.data() : nullptr, n ? v.data() : nullptr, un));
    if (!k.materials.empty())
      must(mpm_set_materials(sim, k.materials.data(), (uint32_t)k.materials.size(), ids.data(), un));
    else
      must(mpm_set_materials(sim, &sim->cfg.rheology, 1, ids.data(), un));
    if (n) {
      must(mpm_set_particle_mass_volume(sim, mass.data(), vol.data(), un));
      must(mpm_write_particle_state(sim, C.data(), F.data(), jp.data(), un));
    }
    if (k.materials.empty()) sim->rows.clear();
    sim->invalidate();
  });
}

int mpm_sim64_create(mpm_engine* engine, const mpm_config* cfg, mpm_sim64** out) {
  return guard([&] {
    REQUIRE(engine && engine->e && cfg && out, MPM_ERR_INVALID, "null argument");
    validate_config(*cfg);
    REQUIRE(cfg->time_step == MPM_TIME_STEP_EXPLICIT, MPM_ERR_UNSUPPORTED,
            "the all-FP64 simulation runs the explicit step only");
    engine->e->check();
    auto s = std::make_unique<mpm_sim64>();
    s->hold = engine->e;
    s->eng = engine->e.get();
    s->cfg = *cfg;
    mpm::Scene64& sc = s->sc;
    sc.n = (int)cfg->grid_size;
    sc.dx = (double)cfg->cell_size;
    sc.inv_dx = (double)(1.0f / cfg->cell_size);  // f32 1/dx from the host, as the reference (mpm.rs:2389)
    for (int a = 0; a < 3; ++a) {
      sc.o[a] = (double)cfg->grid_origin[a];
      sc.win[a] = cfg->grid_window_cells[a];
    }
    sc.gy = (double)cfg->gravity_y;
    sc.friction = (double)cfg->boundary_friction;
    sc.pad = cfg->boundary_pad ? (int)cfg->boundary_pad : 2;
    sc.sticky = cfg->walls == MPM_WALLS_STICKY ? 1 : 0;
    for (int a = 0; a < 3; ++a) {
      sc.lo[a] = sc.o[a] + (double)(sc.win[a] + sc.pad) * sc.dx;
      sc.hi[a] = sc.o[a] + (double)(sc.win[a] + (sc.n - sc.pad - 1)) * sc.dx;
    }
    sc.tol = 1.0e-14;
    sc.sweeps = 30;
    s->set_rows(&cfg->rheology, 1);
    const size_t n3 = (size_t)sc.n * sc.n * sc.n;
    s->gmass.alloc(n3);
    s->gmom.alloc(3 * n3);
    s->gvel.alloc(3 * n3);
    s->totals.alloc(4);
    s->status.alloc(4);
    MPM_CK(cudaMemsetAsync(s->status.ptr, 0, 16, s->eng->stream));
    MPM_CK(cudaMemsetAsync(s->gmass.ptr, 0, n3 * 8, s->eng->stream));
    MPM_CK(cudaMemsetAsync(s->gmom.ptr, 0, 3 * n3 * 8, s->eng->stream));
    *out = s.release();
  });
}

int mpm_sim64_destroy(mpm_sim64* sim) {
  return guard([&] { delete sim; });
}

int mpm_sim64_set_particles(mpm_sim64* sim, const double* xyz, uint32_t n) {
  return guard([&] {
    REQUIRE(sim && (xyz || n == 0), MPM_ERR_INVALID, "null argument");
    REQUIRE(n <= sim->cfg.max_particles || sim->cfg.max_particles == 0, MPM_ERR_INVALID,
            "particle count exceeds max_particles");
    for (size_t i = 0; i < 3 * (size_t)n; ++i)
      REQUIRE(std::isfinite(xyz[i]), MPM_ERR_INVALID, "MPM particle positions must be finite");
    sim->count = n;
    const size_t m = n ? n : 1;
    sim->pos.alloc(3 * m);
    sim->vel.alloc(3 * m);
    sim->C.alloc(9 * m);
    sim->F.alloc(9 * m);
    sim->mass.alloc(m);
    sim->vol.alloc(m);
    sim->jp.alloc(m);
    sim->mat.alloc(m);
    std::vector<double> F(9 * m, 0.0), mass(m, (double)sim->cfg.particle_mass), vol(m, (double)sim->cfg.particle_volume);
    for (size_t i = 0; i < m; ++i) F[9 * i] = F[9 * i + 4] = F[9 * i + 8] = 1.0;
    cudaStream_t st = sim->eng->stream;
    if (n) MPM_CK(cudaMemcpyAsync(sim->pos.ptr, xyz, 3 * (size_t)n * 8, cudaMemcpyHostToDevice, st));
    MPM_CK(cudaMemsetAsync(sim->vel.ptr, 0, 3 * m * 8, st));
    MPM_CK(cudaMemsetAsync(sim->C.ptr, 0, 9 * m * 8, st));
    MPM_CK(cudaMemsetAsync(sim->jp.ptr, 0, m * 8, st));
    MPM_CK(cudaMemsetAsync(sim->mat.ptr, 0, m * 4, st));
    MPM_CK(cudaMemcpyAsync(sim->F.ptr, F.data(), F.size() * 8, cudaMemcpyHostToDevice, st));
    MPM_CK(cudaMemcpyAsync(sim->mass.ptr, mass.data(), m * 8, cudaMemcpyHostToDevice, st));
    MPM_CK(cudaMemcpyAsync(sim->vol.ptr, vol.data(), m * 8, cudaMemcpyHostToDevice, st));
    MPM_CK(cudaMemsetAsync(sim->status.ptr, 0, 16, st));
    MPM_CK(cudaStreamSynchronize(st));
  });
}

int mpm_sim64_set_materials(mpm_sim64* sim, const mpm_rheology* rows, uint32_t n_rows, const uint32_t* ids,
                            uint32_t n) {
  return guard([&] {
    REQUIRE(sim && rows && n_rows >= 1 && n_rows <= 8, MPM_ERR_INVALID, "MPM materials need 1..8 rows");
    REQUIRE(n == sim->count && (ids || n == 0), MPM_ERR_INVALID, "material ids must cover every particle");
    for (uint32_t i = 0; i < n; ++i) REQUIRE(ids[i] < n_rows, MPM_ERR_INVALID, "material id out of range");
    for (uint32_t r = 0; r < n_rows; ++r) REQUIRE(rows[r].kind <= MPM_RHEOLOGY_VISCOUS, MPM_ERR_INVALID, "unknown MPM rheology");
    sim->set_rows(rows, n_rows);
    if (n) {
      MPM_CK(cudaMemcpyAsync(sim->mat.ptr, ids, (size_t)n * 4, cudaMemcpyHostToDevice, sim->eng->stream));
      MPM_CK(cudaStreamSynchronize(sim->eng->stream));
    }
  });
}

int mpm_sim64_step_n(mpm_sim64* sim, double dt, uint32_t substeps) {
  return guard([&] {
    REQUIRE(sim, MPM_ERR_INVALID, "null simulation");
    REQUIRE(std::isfinite(dt) && dt > 0.0, MPM_ERR_INVALID, "MPM dt must be finite and > 0");
    sim->eng->check();
    sim->sc.dt = dt;
    sim->sc.gy = (double)sim->cfg.gravity_y;
    MPM_CK(mpm::launch_step64(sim->sc, sim->state(), substeps, sim->eng->stream));
    sim->eng->launches += (uint64_t)substeps * 4;
  });
}

int mpm_sim64_read_state(mpm_sim64* sim, double* pos, double* vel, double* F, uint32_t cap, uint32_t* count_out) {
  return guard([&] {
    REQUIRE(sim, MPM_ERR_INVALID, "null simulation");
    const uint32_t n = std::min(cap, sim->count);
    cudaStream_t st = sim->eng->stream;
    if (pos && n) MPM_CK(cudaMemcpyAsync(pos, sim->pos.ptr, 3 * (size_t)n * 8, cudaMemcpyDeviceToHost, st));
    if (vel && n) MPM_CK(cudaMemcpyAsync(vel, sim->vel.ptr, 3 * (size_t)n * 8, cudaMemcpyDeviceToHost, st));
    if (F && n) MPM_CK(cudaMemcpyAsync(F, sim->F.ptr, 9 * (size_t)n * 8, cudaMemcpyDeviceToHost, st));
    MPM_CK(cudaStreamSynchronize(st));
    if (count_out) *count_out = n;
  });
}

int mpm_sim64_grid_totals(mpm_sim64* sim, double* out4) {
  return guard([&] {
    REQUIRE(sim && out4, MPM_ERR_INVALID, "null argument");
    MPM_CK(mpm::launch_totals64(sim->sc, sim->state(), sim->totals.ptr, sim->eng->stream));
    MPM_CK(cudaMemcpyAsync(out4, sim->totals.ptr, 32, cudaMemcpyDeviceToHost, sim->eng->stream));
    MPM_CK(cudaStreamSynchronize(sim->eng->stream));
  });
}

int mpm_sim64_read_status(mpm_sim64* sim, mpm_status_info* out) {
  return guard([&] {
    REQUIRE(sim && out, MPM_ERR_INVALID, "null argument");
    uint32_t w[4];
    MPM_CK(cudaMemcpyAsync(w, sim->status.ptr, 16, cudaMemcpyDeviceToHost, sim->eng->stream));
    MPM_CK(cudaStreamSynchronize(sim->eng->stream));
    out->numerical_fault = (w[0] & 2u) ? 1u : 0u;
    out->completed_substeps = w[1];
    out->fault_bits = w[0];
    out->active_tiles = 0;
  });
}

int mpm_server_stats_get(mpm_server* server, mpm_server_stats* out) {
  return guard([&] {
    REQUIRE(server && out, MPM_ERR_INVALID, "null argument");
    out->admitted = server->admitted;
    out->completed = server->completed;
    out->resident_scenes = server->g->live_scenes();
    out->resident_bytes = server->resident;
    out->particle_steps = server->particle_steps;
    out->tick_ms_p50 = pct(server->tick_ms, 0.5);
    out->tick_ms_p99 = pct(server->tick_ms, 0.99);
    out->queue_ms_p50 = pct(server->queue_ms, 0.5);
    out->queue_ms_p99 = pct(server->queue_ms, 0.99);
    out->admit_ms = server->admit_ms;
    out->step_ms = server->step_ms;
    out->retire_ms = server->retire_ms;
    out->ticks = server->ticks;
    out->faulted = server->faulted;
    out->graph_builds = server->g->graph_builds;
    out->graph_build_ms = server->g->graph_build_ms;
  });
}

}  // extern "C"
