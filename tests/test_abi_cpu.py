"""CPU checks of the C ABI: the library loads, exports every declared symbol,
and its host-side logic (presets, material constants, argument validation,
errors) behaves like the reference without touching a GPU."""

import ctypes
import math
import re
from pathlib import Path

import numpy as np
import pytest

import molla_b200 as m
from molla_b200 import _ffi
from oracle import oracle as O

ROOT = Path(__file__).resolve().parent.parent


def declared_symbols():
    text = (ROOT / "include" / "molla_mpm.h").read_text()
    return sorted(set(re.findall(r"^MPM_API\s+[\w\s\*]+?\b(mpm_\w+)\s*\(", text, re.M)))


def test_library_exports_every_declared_symbol():
    L = ctypes.CDLL(str(_ffi.LIB_PATH))
    syms = declared_symbols()
    assert len(syms) >= 50
    missing = [s for s in syms if not hasattr(L, s)]
    assert not missing, missing
    # and the Python binding covers them all
    assert set(syms) == set(_ffi.SIGNATURES), set(syms) ^ set(_ffi.SIGNATURES)


def test_rust_binding_covers_every_declared_symbol():
    """The Rust extern "C" declarations a molla maintainer adds to
    molla-solvers (molla_b200/ffi/mpm_b200_ffi.rs) name every entry point of
    the header with its argument count."""
    hdr = re.sub(r"/\*.*?\*/", "", (ROOT / "include" / "molla_mpm.h").read_text(), flags=re.S)
    arity = {}
    for name, args in re.findall(r"MPM_API\s+[\w\s\*]+?\b(mpm_\w+)\s*\(([^)]*)\)\s*;", hdr):
        arity[name] = len([a for a in args.split(",") if a.strip() and a.strip() != "void"])
    src = re.sub(r"//[^\n]*", "", (ROOT / "molla_b200" / "ffi" / "mpm_b200_ffi.rs").read_text())
    bound = {}
    for name, args in re.findall(r"pub fn (mpm_\w+)\(([^)]*)\)", src, flags=re.S):
        bound[name] = len([a for a in args.split(",") if a.strip()])
    assert set(arity) == set(declared_symbols())
    assert set(bound) == set(arity), set(bound) ^ set(arity)
    assert {k: v for k, v in bound.items() if arity[k] != v} == {}


def header_structs():
    """Field names, in order, of every `typedef struct X { ... } X;` of the
    header (array fields by name)."""
    hdr = re.sub(r"/\*.*?\*/", "", (ROOT / "include" / "molla_mpm.h").read_text(), flags=re.S)
    out = {}
    for name, body in re.findall(r"typedef struct (mpm_\w+)\s*\{(.*?)\}\s*\1\s*;", hdr, flags=re.S):
        fields = []
        for decl in body.split(";"):
            decl = decl.strip()
            if not decl:
                continue
            # "T a, b[3]" declares a and b: the last identifier of each part
            for part in decl.split(","):
                fields.append(re.findall(r"(\w+)\s*(?:\[[^\]]*\])?\s*$", part.strip())[0])
        out[name] = fields
    return out


def test_struct_fields_match_across_header_ctypes_and_rust():
    """Every struct of the header has the same fields in the same order in
    the ctypes mirror (molla_b200/_ffi.py) and in the Rust #[repr(C)]
    mirror (molla_b200/ffi/mpm_b200_ffi.rs), so that a field added to the
    header cannot be left out of a binding."""
    hdr = header_structs()
    assert {"mpm_config", "mpm_rheology", "mpm_status_info", "mpm_server_stats", "mpm_shapes"} <= set(hdr)
    src = re.sub(r"//[^\n]*", "", (ROOT / "molla_b200" / "ffi" / "mpm_b200_ffi.rs").read_text())
    rust = {name: re.findall(r"pub (\w+)\s*:", body)
            for name, body in re.findall(r"pub struct (mpm_\w+)\s*\{(.*?)\}", src, flags=re.S)}
    for name, fields in hdr.items():
        cls = getattr(_ffi, name, None)
        if cls is not None:
            assert [f[0] for f in cls._fields_] == fields, name
        assert rust.get(name) == fields, (name, rust.get(name), fields)


def test_abi_version_and_error_channel():
    L = _ffi.lib()
    assert L.mpm_abi_version() == 1
    rc = L.mpm_sim_destroy(None)
    assert rc == 0
    c = _ffi.mpm_config()
    assert L.mpm_config_preset(99, ctypes.byref(c)) == _ffi.MPM_ERR_INVALID
    assert "preset" in _ffi.last_error()


def test_presets_match_reference():
    sand = m.MpmConfig.sand()  # mpm.rs:540-560
    assert sand.grid_size == 32 and math.isclose(sand.cell_size, 0.05, rel_tol=1e-7)
    assert math.isclose(sand.youngs, 5e3) and math.isclose(sand.poisson, 0.3, rel_tol=1e-7)
    assert sand.rheology.kind == 0 and math.isclose(sand.rheology.friction_angle, math.radians(30), rel_tol=1e-6)
    snow = m.MpmConfig.snow()  # mpm.rs:609-631
    assert snow.rheology.kind == 1 and math.isclose(snow.rheology.theta_c, 0.025, rel_tol=1e-6)
    assert math.isclose(snow.rheology.hardening, 10.0) and math.isclose(snow.youngs, 1.4e5)
    visc = m.MpmConfig.viscous()  # mpm.rs:637-655
    assert visc.rheology.kind == 2 and visc.rheology.velocity_damping == 4.0 and visc.rheology.affine_damping == 8.0
    cal = m.MpmConfig.sand_calibrated()
    assert cal.grid_size == 48 and cal.time_step == m.MpmTimeStep.IMPLICIT


def test_dp_alpha_matches_oracle_material_row():
    L = _ffi.lib()
    for phi in (0.0, 0.1, 0.5, math.radians(30), 1.2):
        assert L.mpm_dp_alpha(phi) == O.lib().orc_dp_alpha_f32(phi)


def test_engine_without_gpu_reports_gpu_error():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(m.GpuError):
        m.Engine(0)


def test_struct_layout_matches_c_header(tmp_path):
    """The ctypes mirror (and any Rust #[repr(C)] mirror) must match the C
    header: compile the header with the C compiler and compare sizes/offsets."""
    import shutil
    import subprocess
    cc = shutil.which("gcc") or "/usr/bin/gcc"
    src = tmp_path / "layout.c"
    src.write_text(
        '#include <stdio.h>\n#include <stddef.h>\n#include "molla_mpm.h"\n'
        'int main(void){printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\\n", sizeof(mpm_rheology), sizeof(mpm_config),'
        ' sizeof(mpm_status_info), sizeof(mpm_server_stats), offsetof(mpm_config, rheology),'
        ' offsetof(mpm_config, grid_window_cells), sizeof(mpm_render_view), offsetof(mpm_render_view, source),'
        ' offsetof(mpm_render_view, live_position_bytes), sizeof(mpm_sim_info),'
        ' offsetof(mpm_sim_info, max_particles)); return 0;}\n')
    exe = tmp_path / "layout"
    subprocess.run([cc, "-std=c99", f"-I{ROOT / 'include'}", str(src), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    exp = [ctypes.sizeof(_ffi.mpm_rheology), ctypes.sizeof(_ffi.mpm_config), ctypes.sizeof(_ffi.mpm_status_info),
           ctypes.sizeof(_ffi.mpm_server_stats), _ffi.mpm_config.rheology.offset,
           _ffi.mpm_config.grid_window_cells.offset, ctypes.sizeof(_ffi.mpm_render_view),
           _ffi.mpm_render_view.source.offset, _ffi.mpm_render_view.live_position_bytes.offset,
           ctypes.sizeof(_ffi.mpm_sim_info), _ffi.mpm_sim_info.max_particles.offset]
    assert got == exp


def test_render_view_wrapper_exposes_the_live_prefix():
    """MpmParticleRenderView (mpm_render_view.rs:20-36) over a raw view
    struct: count, bytes, source identity and the CUDA array interface of the
    live float4 prefix."""
    raw = _ffi.mpm_render_view(positions=0x7F0000001000, count=3, capacity=10, source=42, live_position_bytes=48)
    v = m.MpmParticleRenderView(raw, owner=None)
    assert v.particle_count() == 3 and v.capacity == 10 and v.live_position_bytes() == 48
    assert v.positions() == 0x7F0000001000
    cai = v.__cuda_array_interface__
    assert cai["shape"] == (3, 4) and cai["typestr"] == "<f4" and cai["data"] == (0x7F0000001000, False)
    assert v.matches_source(m.MpmParticleRenderSource(42))
    assert not v.matches_source(m.MpmParticleRenderSource(43))
    empty = m.MpmParticleRenderView(_ffi.mpm_render_view(positions=0x7F0000001000, count=0, source=42), None)
    assert empty.__cuda_array_interface__["shape"] == (0, 4) and empty.matches_source(v.source())
