// mpm_checkpoint.cuh — the soil checkpoint byte format and its BLAKE3 digest
// (host code).
//
// Format (crates/molla-solvers/src/mpm_checkpoint.rs:71-92, :187-216): the
// 8-byte magic "MOLLSOIL", a little-endian u32 version (1; 2 when the grid
// window is not zero), a 32-byte BLAKE3 digest of everything after the
// 44-byte header (version 2 hashes the version word first), then
// little-endian u32 words: [window x, y, z (version 2)], the configuration
// (grid_size, max_particles, max_rigid, 12 f32 fields, rheology 4 words, time
// step 2 words), the material-row count and rows (4 words each), the particle
// count, and the particle streams one after another: position 4, velocity 4,
// C 12, F 12 (vec4-padded columns), volume 1, mass 1, log-Jp 1, material id
// 1, tire compaction 4 words per particle.  The format is kept word for word
// so that checkpoints move between molla and this library.
#pragma once
#include <cstddef>
#include <cstdint>
#include <vector>

#include "../../include/molla_mpm.h"

namespace mpm {

// BLAKE3 (the published algorithm: 1 KiB chunks, 64-byte blocks, 7-round
// compression, binary tree of chaining values), unkeyed, 32-byte output.
class Blake3 {
 public:
  Blake3();
  void update(const uint8_t* data, size_t len);
  void finalize(uint8_t out[32]) const;

 private:
  struct Output {
    uint32_t cv[8];
    uint32_t block[16];
    uint64_t counter;
    uint32_t block_len;
    uint32_t flags;
  };
  Output chunk_output() const;
  void push_cv(const uint32_t cv[8], uint64_t total_chunks);
  uint32_t cv_[8];
  uint8_t block_[64];
  uint32_t block_len_ = 0;
  uint32_t blocks_done_ = 0;
  uint64_t chunk_counter_ = 0;
  uint32_t stack_[54][8];
  int stack_len_ = 0;
};

struct SoilCheckpoint {
  mpm_config cfg{};                 // reference fields; extensions zero
  int32_t window[3] = {0, 0, 0};
  std::vector<mpm_rheology> materials;  // empty: cfg.rheology is authoritative
  uint32_t count = 0;
  std::vector<uint32_t> words;      // count * 40 words in stream order
};

constexpr int kCheckpointWordsPerParticle = 40;
constexpr int kCheckpointStrides[9] = {4, 4, 12, 12, 1, 1, 1, 1, 4};

std::vector<uint8_t> encode_checkpoint(const SoilCheckpoint& c);
// Rejects corrupt, non-finite, unsupported, oversized and trailing data
// (throws Error with MPM_ERR_INVALID).
SoilCheckpoint decode_checkpoint(const uint8_t* bytes, size_t len, uint32_t max_particles);
// The semantic checks of a checkpoint (configuration, materials, streams).
void validate_checkpoint(const SoilCheckpoint& c);
// Whether two configurations encode to the same configuration words once the
// capacities (max_particles, max_rigid) are ignored (mpm_checkpoint.rs:463-470).
bool checkpoint_config_compatible(const mpm_config& saved, const mpm_config& live);
// Encoded size of a checkpoint with these counts.
size_t checkpoint_bytes(bool lattice, uint32_t material_rows, uint32_t count);

}  // namespace mpm
