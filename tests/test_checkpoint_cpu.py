"""Soil checkpoint byte format and BLAKE3, without a GPU.

The cases follow crates/molla-solvers/src/mpm_checkpoint_tests.rs:3-153
(the `fixture` state, `format_is_lossless_bounded_and_rejects_corruption`,
`valid_digest_does_not_bypass_semantic_validation`).  The bytes are built here
by an independent Python encoder of the format (mpm_checkpoint.rs:71-92,
187-216, 544-619) with the `blake3` package as the digest, and the library
must accept them, re-encode them byte for byte and reject every corruption.
"""

import struct

import numpy as np
import pytest

import molla_b200 as m

blake3 = pytest.importorskip("blake3")

HEADER = 44


def f32(x):
    return struct.unpack("<I", struct.pack("<f", x))[0]


def rheology_words(r):
    kind = r[0]
    if kind == "sand":
        return [0, f32(r[1]), 0, 0]
    if kind == "snow":
        return [1, f32(r[1]), f32(r[2]), f32(r[3])]
    return [2, f32(r[1]), f32(r[2]), 0]


def fixture(count):
    """The reference fixture: sand config (E 1000, 129 particles, 2 rigid), a
    three-row table and `count` particles with distinct stream values."""
    cfg = m.MpmConfig.sand()
    mass, vol = np.float32(cfg.particle_mass), np.float32(cfg.particle_volume)
    streams = []
    for s in range(9):
        for i in range(count):
            f = np.float32(i)
            if s == 0:
                vals = [np.float32(-0.13) + np.float32(i % 7) * np.float32(0.021),
                        np.float32(0.3) + np.float32(i // 7 % 7) * np.float32(0.021),
                        np.float32(-0.07) + np.float32(i // 49) * np.float32(0.021), -0.0]
            elif s == 1:
                vals = [np.float32(0.013) + f * np.float32(0.0001), -0.007, 0.002, 0.0]
            elif s == 2:
                vals = [0.01, 0.002, 0.0, 0.0, 0.0, -0.02, 0.003, 0.0, 0.004, 0.0, 0.008, 0.0]
            elif s == 3:
                vals = [0.97, 0.001, 0.0, 0.0, 0.0, 1.01, 0.002, 0.0, 0.001, 0.0, 0.98, 0.0]
            elif s == 4:
                vals = [vol * (np.float32(1.0) + f * np.float32(0.002))]
            elif s == 5:
                vals = [mass * (np.float32(1.0) + f * np.float32(0.001))]
            elif s == 6:
                vals = [np.float32(-0.1) - f * np.float32(0.001)]
            elif s == 7:
                streams.append(i % 3)
                continue
            else:
                vals = [np.float32(0.005) + f * np.float32(0.00001), np.float32(0.01) + f * np.float32(0.001), 0.02, 3.0]
            streams.extend(f32(float(np.float32(v))) for v in vals)
    return {
        "grid_size": cfg.grid_size, "max_particles": 129, "max_rigid": 2,
        "floats": [cfg.cell_size, *cfg.grid_origin, cfg.gravity_y, 1000.0, cfg.poisson, cfg.friction_angle,
                   cfg.cohesion, cfg.boundary_friction, cfg.particle_mass, cfg.particle_volume],
        "rheology": ("sand", cfg.rheology.friction_angle),
        "time_step": (0, 0),
        "materials": [("sand", 0.5), ("snow", 0.025, 0.0075, 10.0), ("viscous", 3.0, 5.0)],
        "window": (0, 0, 0),
        "count": count,
        "words": streams,
    }


def encode(c):
    lattice = any(c["window"])
    version = 2 if lattice else 1
    w = [v & 0xFFFFFFFF for v in c["window"]] if lattice else []
    w += [c["grid_size"], c["max_particles"], c["max_rigid"]] + [f32(x) for x in c["floats"]]
    w += rheology_words(c["rheology"]) + list(c["time_step"])
    w += [len(c["materials"])]
    for r in c["materials"]:
        w += rheology_words(r)
    w += [c["count"] & 0xFFFFFFFF] + list(c["words"])
    payload = struct.pack(f"<{len(w)}I", *w)
    h = blake3.blake3()
    if version == 2:
        h.update(struct.pack("<I", version))
    h.update(payload)
    return b"MOLLSOIL" + struct.pack("<I", version) + h.digest() + payload


def redigest(b):
    b = bytearray(b)
    b[12:HEADER] = blake3.blake3(bytes(b[HEADER:])).digest()
    return bytes(b)


def rejected(b, maxp=129):
    with pytest.raises(m.MollaError):
        m.checkpoint_reencode(b, maxp)


@pytest.mark.parametrize("n", [0, 1, 63, 64, 65, 1023, 1024, 1025, 2049, 3072, 8193, 65536 + 17, (1 << 20) + 7])
def test_blake3_matches_reference_implementation(n):
    data = np.random.default_rng(n).integers(0, 256, size=n, dtype=np.uint8).tobytes()
    assert m.blake3(data) == blake3.blake3(data).digest()


def test_format_is_lossless_and_bounded():
    for count in (0, 1, 129):
        c = fixture(count)
        for rh in list(c["materials"]):
            c["rheology"] = rh
            for ts in ((0, 0), (1, 3)):
                c["time_step"] = ts
                b = encode(c)
                out, got = m.checkpoint_reencode(b, max(count, 1) if count else 0)
                assert out == b and got == count
                assert len(b) == HEADER + 4 * (21 + 1 + 12 + 1) + count * 160
                if count > 0:
                    rejected(b, count - 1)


def test_lattice_window_uses_version_2():
    c = fixture(1)
    c["window"] = (2, -3, 0)
    b = encode(c)
    assert struct.unpack("<I", b[8:12])[0] == 2
    assert m.checkpoint_reencode(b, 129)[0] == b
    # a version-2 payload with a zero window is rejected even with a valid digest
    z = bytearray(b)
    z[HEADER:HEADER + 12] = bytes(12)
    h = blake3.blake3()
    h.update(struct.pack("<I", 2))
    h.update(bytes(z[HEADER:]))
    z[12:HEADER] = h.digest()
    rejected(bytes(z))


def test_rejects_truncation_bit_flips_and_trailing_data():
    b = encode(fixture(1))
    for n in range(len(b)):
        rejected(b[:n])
    for i in range(len(b)):
        bad = bytearray(b)
        bad[i] ^= 1
        rejected(bytes(bad))
    rejected(redigest(b + bytes(4)))


@pytest.mark.parametrize("mutate", [
    lambda c: c["floats"].__setitem__(0, float("nan")),           # cell size
    lambda c: c.__setitem__("max_particles", 0),
    lambda c: c.__setitem__("grid_size", 0xFFFFFFFF),
    lambda c: c["floats"].__setitem__(6, 0.5),                      # poisson
    lambda c: c.__setitem__("rheology", ("sand", float("inf"))),
    lambda c: c["materials"].__setitem__(1, ("snow", 1.0, 0.0, 1.0)),
    lambda c: c["words"].__setitem__(0, f32(float("nan"))),
    lambda c: c["words"].__setitem__(4, f32(float("inf"))),
    lambda c: c["words"].__setitem__(8, f32(float("nan"))),
    lambda c: c["words"].__setitem__(20, f32(float("inf"))),
    lambda c: c["words"].__setitem__(32, 0),                        # volume 0
    lambda c: c["words"].__setitem__(33, f32(-1.0)),                # negative mass
    lambda c: c["words"].__setitem__(34, f32(float("nan"))),        # log-Jp
    lambda c: c["words"].__setitem__(35, 3),                        # material id outside the table
    lambda c: c["words"].__setitem__(36, f32(float("nan"))),        # tire compaction
    lambda c: c.__setitem__("count", 0xFFFFFFFF),
    lambda c: c["words"].pop(),
    lambda c: c.__setitem__("materials", [c["rheology"]] * 9),
])
def test_valid_digest_does_not_bypass_semantic_validation(mutate):
    c = fixture(1)
    mutate(c)
    rejected(encode(c))


@pytest.mark.parametrize("index", [15, 19])
def test_unsupported_rheology_or_time_step_encoding(index):
    b = bytearray(encode(fixture(1)))
    b[HEADER + 4 * index:HEADER + 4 * index + 4] = struct.pack("<I", 99)
    rejected(redigest(bytes(b)))
