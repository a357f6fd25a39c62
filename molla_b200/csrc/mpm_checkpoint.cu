// mpm_checkpoint.cu — soil checkpoint encode/decode and BLAKE3 (host code).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>

#include "mpm_checkpoint.cuh"
#include "mpm_runtime.cuh"

namespace mpm {

// ---------------------------------------------------------------------------
// BLAKE3, restated from the published specification (O'Connor, Aumasson,
// Neves, Wilcox-O'Hearn, 2020): the compression function is 7 rounds of the
// ChaCha-style quarter-round G over a 4x4 word state, with the message words
// permuted between rounds; chunks of 1024 bytes are compressed block by block
// (64 bytes) with CHUNK_START / CHUNK_END flags; chunk chaining values are
// merged pairwise into parent nodes; the root is compressed with ROOT.
namespace {

constexpr uint32_t kIv[8] = {0x6A09E667u, 0xBB67AE85u, 0x3C6EF372u, 0xA54FF53Au,
                             0x510E527Fu, 0x9B05688Cu, 0x1F83D9ABu, 0x5BE0CD19u};
constexpr int kPerm[16] = {2, 6, 3, 10, 7, 0, 4, 13, 1, 11, 12, 5, 9, 14, 15, 8};
constexpr uint32_t kChunkStart = 1u, kChunkEnd = 2u, kParent = 4u, kRoot = 8u;
constexpr size_t kChunkLen = 1024, kBlockLen = 64;

inline uint32_t rotr(uint32_t x, int n) { return (x >> n) | (x << (32 - n)); }

inline void g(uint32_t* s, int a, int b, int c, int d, uint32_t mx, uint32_t my) {
  s[a] = s[a] + s[b] + mx;
  s[d] = rotr(s[d] ^ s[a], 16);
  s[c] = s[c] + s[d];
  s[b] = rotr(s[b] ^ s[c], 12);
  s[a] = s[a] + s[b] + my;
  s[d] = rotr(s[d] ^ s[a], 8);
  s[c] = s[c] + s[d];
  s[b] = rotr(s[b] ^ s[c], 7);
}

// Full 16-word output of one compression.
void compress(const uint32_t cv[8], const uint32_t block[16], uint64_t counter, uint32_t block_len, uint32_t flags,
              uint32_t out[16]) {
  uint32_t s[16] = {cv[0], cv[1], cv[2], cv[3], cv[4], cv[5], cv[6], cv[7],
                    kIv[0], kIv[1], kIv[2], kIv[3], (uint32_t)counter, (uint32_t)(counter >> 32), block_len, flags};
  uint32_t m[16];
  std::memcpy(m, block, sizeof(m));
  for (int r = 0; r < 7; ++r) {
    g(s, 0, 4, 8, 12, m[0], m[1]);
    g(s, 1, 5, 9, 13, m[2], m[3]);
    g(s, 2, 6, 10, 14, m[4], m[5]);
    g(s, 3, 7, 11, 15, m[6], m[7]);
    g(s, 0, 5, 10, 15, m[8], m[9]);
    g(s, 1, 6, 11, 12, m[10], m[11]);
    g(s, 2, 7, 8, 13, m[12], m[13]);
    g(s, 3, 4, 9, 14, m[14], m[15]);
    if (r < 6) {
      uint32_t t[16];
      for (int i = 0; i < 16; ++i) t[i] = m[kPerm[i]];
      std::memcpy(m, t, sizeof(m));
    }
  }
  for (int i = 0; i < 8; ++i) {
    out[i] = s[i] ^ s[i + 8];
    out[i + 8] = s[i + 8] ^ cv[i];
  }
}

void words_of(const uint8_t* b, uint32_t w[16]) {
  for (int i = 0; i < 16; ++i)
    w[i] = (uint32_t)b[4 * i] | ((uint32_t)b[4 * i + 1] << 8) | ((uint32_t)b[4 * i + 2] << 16) |
           ((uint32_t)b[4 * i + 3] << 24);
}

void parent_cv(const uint32_t left[8], const uint32_t right[8], uint32_t out[8]) {
  uint32_t block[16], full[16];
  std::memcpy(block, left, 32);
  std::memcpy(block + 8, right, 32);
  compress(kIv, block, 0, (uint32_t)kBlockLen, kParent, full);
  std::memcpy(out, full, 32);
}

}  // namespace

Blake3::Blake3() {
  std::memcpy(cv_, kIv, sizeof(cv_));
  std::memset(block_, 0, sizeof(block_));
}

// The last block of the current chunk, ready to be compressed as a chunk
// output (CHUNK_END, plus CHUNK_START if it is the chunk's only block).
Blake3::Output Blake3::chunk_output() const {
  Output o;
  std::memcpy(o.cv, cv_, sizeof(cv_));
  uint8_t padded[64] = {0};
  std::memcpy(padded, block_, block_len_);
  words_of(padded, o.block);
  o.counter = chunk_counter_;
  o.block_len = block_len_;
  o.flags = kChunkEnd | (blocks_done_ == 0 ? kChunkStart : 0u);
  return o;
}

void Blake3::push_cv(const uint32_t cv[8], uint64_t total_chunks) {
  uint32_t cur[8];
  std::memcpy(cur, cv, 32);
  while ((total_chunks & 1) == 0) {
    uint32_t merged[8];
    parent_cv(stack_[--stack_len_], cur, merged);
    std::memcpy(cur, merged, 32);
    total_chunks >>= 1;
  }
  std::memcpy(stack_[stack_len_++], cur, 32);
}

void Blake3::update(const uint8_t* data, size_t len) {
  while (len > 0) {
    // A full chunk is closed only when more input follows it.
    if (blocks_done_ * kBlockLen + block_len_ == kChunkLen) {
      const Output o = chunk_output();
      uint32_t full[16];
      compress(o.cv, o.block, o.counter, o.block_len, o.flags, full);
      push_cv(full, chunk_counter_ + 1);
      ++chunk_counter_;
      std::memcpy(cv_, kIv, sizeof(cv_));
      blocks_done_ = 0;
      block_len_ = 0;
    }
    // A full block is compressed only when more input follows it.
    if (block_len_ == kBlockLen) {
      uint32_t w[16], full[16];
      words_of(block_, w);
      compress(cv_, w, chunk_counter_, (uint32_t)kBlockLen, blocks_done_ == 0 ? kChunkStart : 0u, full);
      std::memcpy(cv_, full, sizeof(cv_));
      ++blocks_done_;
      block_len_ = 0;
    }
    const size_t take = std::min(len, kBlockLen - block_len_);
    std::memcpy(block_ + block_len_, data, take);
    block_len_ += (uint32_t)take;
    data += take;
    len -= take;
  }
}

void Blake3::finalize(uint8_t out[32]) const {
  Output o = chunk_output();
  for (int i = stack_len_ - 1; i >= 0; --i) {
    uint32_t full[16], cv[8];
    compress(o.cv, o.block, o.counter, o.block_len, o.flags, full);
    std::memcpy(cv, full, 32);
    Output p;
    std::memcpy(p.cv, kIv, 32);
    std::memcpy(p.block, stack_[i], 32);
    std::memcpy(p.block + 8, cv, 32);
    p.counter = 0;
    p.block_len = (uint32_t)kBlockLen;
    p.flags = kParent;
    o = p;
  }
  uint32_t full[16];
  compress(o.cv, o.block, 0, o.block_len, o.flags | kRoot, full);
  for (int i = 0; i < 8; ++i) {
    out[4 * i] = (uint8_t)full[i];
    out[4 * i + 1] = (uint8_t)(full[i] >> 8);
    out[4 * i + 2] = (uint8_t)(full[i] >> 16);
    out[4 * i + 3] = (uint8_t)(full[i] >> 24);
  }
}

// ---------------------------------------------------------------------------
// Soil checkpoint (crates/molla-solvers/src/mpm_checkpoint.rs).
namespace {

constexpr char kMagic[8] = {'M', 'O', 'L', 'L', 'S', 'O', 'I', 'L'};
constexpr uint32_t kVersion = 1, kLatticeVersion = 2;
constexpr size_t kHeaderBytes = 44;

[[noreturn]] void bad(const std::string& what) { throw Error(MPM_ERR_INVALID, "MPM soil checkpoint: " + what); }

uint32_t bits(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  return u;
}
float flt(uint32_t u) {
  float f;
  std::memcpy(&f, &u, 4);
  return f;
}

// mpm_checkpoint.rs:544-557: kind, then the kind's three parameters.
void rheology_words(const mpm_rheology& r, std::vector<uint32_t>& w) {
  switch (r.kind) {
    case MPM_RHEOLOGY_SAND: w.insert(w.end(), {0u, bits(r.friction_angle), 0u, 0u}); break;
    case MPM_RHEOLOGY_SNOW: w.insert(w.end(), {1u, bits(r.theta_c), bits(r.theta_s), bits(r.hardening)}); break;
    default: w.insert(w.end(), {2u, bits(r.velocity_damping), bits(r.affine_damping), 0u}); break;
  }
}

// mpm_checkpoint.rs:594-619.
void config_words(const mpm_config& c, std::vector<uint32_t>& w) {
  w.insert(w.end(), {c.grid_size, c.max_particles, c.max_rigid});
  for (float f : {c.cell_size, c.grid_origin[0], c.grid_origin[1], c.grid_origin[2], c.gravity_y, c.youngs, c.poisson,
                  c.friction_angle, c.cohesion, c.boundary_friction, c.particle_mass, c.particle_volume})
    w.push_back(bits(f));
  rheology_words(c.rheology, w);
  if (c.time_step == MPM_TIME_STEP_EXPLICIT) w.insert(w.end(), {0u, 0u});
  else w.insert(w.end(), {1u, c.jacobi_iters});
}

void digest(uint32_t version, const uint8_t* payload, size_t len, uint8_t out[32]) {
  Blake3 h;
  if (version == kLatticeVersion) {
    const uint8_t v[4] = {(uint8_t)version, (uint8_t)(version >> 8), (uint8_t)(version >> 16), (uint8_t)(version >> 24)};
    h.update(v, 4);
  }
  h.update(payload, len);
  h.finalize(out);
}

struct Reader {
  const uint32_t* p;
  size_t left;
  uint32_t next() {
    if (!left) bad("truncated metadata");
    --left;
    return *p++;
  }
  float f() { return flt(next()); }
  mpm_rheology rheology() {
    mpm_rheology r{};
    const uint32_t kind = next();
    const uint32_t a = next(), b = next(), c = next();
    if (kind == 0 && b == 0 && c == 0) {
      r.kind = MPM_RHEOLOGY_SAND;
      r.friction_angle = flt(a);
    } else if (kind == 1) {
      r.kind = MPM_RHEOLOGY_SNOW;
      r.theta_c = flt(a);
      r.theta_s = flt(b);
      r.hardening = flt(c);
    } else if (kind == 2 && c == 0) {
      r.kind = MPM_RHEOLOGY_VISCOUS;
      r.velocity_damping = flt(a);
      r.affine_damping = flt(b);
    } else {
      bad("unsupported or noncanonical rheology encoding");
    }
    return r;
  }
};

bool rheology_valid(const mpm_rheology& r) {
  switch (r.kind) {
    case MPM_RHEOLOGY_SAND: return std::isfinite(r.friction_angle) && r.friction_angle >= 0.f && r.friction_angle < 1.57079632679f;
    case MPM_RHEOLOGY_SNOW:
      return std::isfinite(r.theta_c) && r.theta_c >= 0.f && r.theta_c < 1.f && std::isfinite(r.theta_s) &&
             r.theta_s >= 0.f && std::isfinite(r.hardening) && r.hardening >= 0.f;
    case MPM_RHEOLOGY_VISCOUS:
      return std::isfinite(r.velocity_damping) && r.velocity_damping >= 0.f && std::isfinite(r.affine_damping) &&
             r.affine_damping >= 0.f;
    default: return false;
  }
}

}  // namespace

void validate_checkpoint(const SoilCheckpoint& k) {
  const mpm_config& c = k.cfg;
  // grid_size^3 must fit in u32 (1625^3 < 2^32 <= 1626^3)
  const bool ok = c.grid_size > 0 && c.grid_size <= 1625u && c.max_particles > 0 && c.max_rigid > 0 &&
                  k.count <= c.max_particles && std::isfinite(c.cell_size) && c.cell_size > 0.f &&
                  std::isfinite(c.grid_origin[0]) && std::isfinite(c.grid_origin[1]) && std::isfinite(c.grid_origin[2]) &&
                  std::isfinite(c.gravity_y) && std::isfinite(c.youngs) && c.youngs >= 0.f && std::isfinite(c.poisson) &&
                  c.poisson > -1.f && c.poisson < 0.5f && std::isfinite(c.friction_angle) &&
                  std::isfinite(c.cohesion) && c.cohesion >= 0.f && std::isfinite(c.boundary_friction) &&
                  c.boundary_friction >= 0.f && c.boundary_friction <= 1.f && std::isfinite(c.particle_mass) &&
                  c.particle_mass > 0.f && std::isfinite(c.particle_volume) && c.particle_volume > 0.f &&
                  k.materials.size() <= 8 && k.words.size() == (size_t)k.count * kCheckpointWordsPerParticle;
  if (!ok) bad("invalid configuration or state length");
  if (!rheology_valid(c.rheology)) bad("invalid material parameters");
  for (const mpm_rheology& r : k.materials)
    if (!rheology_valid(r)) bad("invalid material parameters");
  size_t off = 0;
  for (int s = 0; s < 9; ++s) {
    const size_t len = (size_t)kCheckpointStrides[s] * k.count;
    if (s == 7) {
      const uint32_t rows = (uint32_t)std::max<size_t>(k.materials.size(), 1);
      for (size_t i = 0; i < len; ++i)
        if (k.words[off + i] >= rows) bad("material ID outside authoritative table");
    } else {
      for (size_t i = 0; i < len; ++i) {
        const float v = flt(k.words[off + i]);
        if (!std::isfinite(v) || ((s == 4 || s == 5) && v <= 0.f))
          bad("non-finite history or nonpositive mass/reference volume");
      }
    }
    off += len;
  }
}

bool checkpoint_config_compatible(const mpm_config& saved, const mpm_config& live) {
  mpm_config a = saved;
  a.max_particles = live.max_particles;
  a.max_rigid = live.max_rigid;
  std::vector<uint32_t> wa, wb;
  config_words(a, wa);
  config_words(live, wb);
  return wa == wb;
}

size_t checkpoint_bytes(bool lattice, uint32_t material_rows, uint32_t count) {
  return kHeaderBytes + 4 * ((lattice ? 3u : 0u) + 21u + 1u + 4u * (size_t)material_rows + 1u +
                             (size_t)kCheckpointWordsPerParticle * count);
}

std::vector<uint8_t> encode_checkpoint(const SoilCheckpoint& k) {
  const bool lattice = k.window[0] != 0 || k.window[1] != 0 || k.window[2] != 0;
  const uint32_t version = lattice ? kLatticeVersion : kVersion;
  std::vector<uint32_t> w;
  w.reserve(40 + k.words.size());
  if (lattice) w.insert(w.end(), {(uint32_t)k.window[0], (uint32_t)k.window[1], (uint32_t)k.window[2]});
  config_words(k.cfg, w);
  w.push_back((uint32_t)k.materials.size());
  for (const mpm_rheology& r : k.materials) rheology_words(r, w);
  w.push_back(k.count);
  w.insert(w.end(), k.words.begin(), k.words.end());
  std::vector<uint8_t> out(kHeaderBytes + 4 * w.size());
  std::memcpy(out.data(), kMagic, 8);
  for (int i = 0; i < 4; ++i) out[8 + i] = (uint8_t)(version >> (8 * i));
  for (size_t i = 0; i < w.size(); ++i)
    for (int b = 0; b < 4; ++b) out[kHeaderBytes + 4 * i + b] = (uint8_t)(w[i] >> (8 * b));
  digest(version, out.data() + kHeaderBytes, out.size() - kHeaderBytes, out.data() + 12);
  return out;
}

SoilCheckpoint decode_checkpoint(const uint8_t* bytes, size_t len, uint32_t max_particles) {
  if (len < kHeaderBytes) bad("truncated checkpoint header");
  const uint32_t version = (uint32_t)bytes[8] | ((uint32_t)bytes[9] << 8) | ((uint32_t)bytes[10] << 16) |
                           ((uint32_t)bytes[11] << 24);
  // mpm_checkpoint.rs:78-82: header + (23 + 4 * 8 + 40 max_particles) words.
  const uint64_t max_bytes = kHeaderBytes + (23ull + 32ull + 40ull * max_particles) * 4ull +
                             (version == kLatticeVersion ? 12ull : 0ull);
  uint8_t d[32];
  bool ok = (version == kVersion || version == kLatticeVersion) && len <= max_bytes &&
            std::memcmp(bytes, kMagic, 8) == 0 && (len - kHeaderBytes) % 4 == 0;
  if (ok) {
    digest(version, bytes + kHeaderBytes, len - kHeaderBytes, d);
    ok = std::memcmp(d, bytes + 12, 32) == 0;
  }
  if (!ok) bad("invalid format, digest or allocation limit");
  std::vector<uint32_t> words((len - kHeaderBytes) / 4);
  for (size_t i = 0; i < words.size(); ++i) {
    const uint8_t* b = bytes + kHeaderBytes + 4 * i;
    words[i] = (uint32_t)b[0] | ((uint32_t)b[1] << 8) | ((uint32_t)b[2] << 16) | ((uint32_t)b[3] << 24);
  }
  Reader r{words.data(), words.size()};
  SoilCheckpoint k;
  if (version == kLatticeVersion) {
    for (int a = 0; a < 3; ++a) k.window[a] = (int32_t)r.next();
    if (k.window[0] == 0 && k.window[1] == 0 && k.window[2] == 0) bad("zero-offset checkpoints use version 1");
  }
  mpm_config& c = k.cfg;
  c.grid_size = r.next();
  c.max_particles = r.next();
  c.max_rigid = r.next();
  c.cell_size = r.f();
  for (int a = 0; a < 3; ++a) c.grid_origin[a] = r.f();
  c.gravity_y = r.f();
  c.youngs = r.f();
  c.poisson = r.f();
  c.friction_angle = r.f();
  c.cohesion = r.f();
  c.boundary_friction = r.f();
  c.particle_mass = r.f();
  c.particle_volume = r.f();
  c.rheology = r.rheology();
  const uint32_t kind = r.next(), iters = r.next();
  if (kind == 0 && iters == 0) {
    c.time_step = MPM_TIME_STEP_EXPLICIT;
  } else if (kind == 1) {
    c.time_step = MPM_TIME_STEP_IMPLICIT;
    c.jacobi_iters = iters;
  } else {
    bad("unsupported time step encoding");
  }
  for (int a = 0; a < 3; ++a) c.grid_window_cells[a] = k.window[a];
  const uint32_t rows = r.next();
  if (rows > 8) bad("material table exceeds capacity");
  for (uint32_t i = 0; i < rows; ++i) k.materials.push_back(r.rheology());
  k.count = r.next();
  if (k.count > max_particles || r.left != (size_t)k.count * kCheckpointWordsPerParticle)
    bad("particle count or payload length mismatch");
  k.words.assign(r.p, r.p + r.left);
  validate_checkpoint(k);
  return k;
}

}  // namespace mpm
