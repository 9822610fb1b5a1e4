"""CPU tests of the C ABI boundary: the shared library loads, exports every symbol include/dfsph_c.h
declares, the ctypes layouts match the header, and without a GPU the product fails loudly."""
import ctypes as C
import re
import shutil
import subprocess
from pathlib import Path

import pytest

from splishsplash_for_cuda_b200 import _capi

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols():
    text = (ROOT / "include" / "dfsph_c.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(dfsph_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_bound_symbols():
    syms = declared_symbols()
    assert len(syms) >= 20
    assert set(syms) == set(_capi.SIGNATURES), set(syms) ^ set(_capi.SIGNATURES)


def test_library_exports_every_declared_symbol(cuda_lib):
    for name in declared_symbols():
        assert hasattr(cuda_lib, name), name


def test_checked_library_exports_every_declared_symbol():
    """The range-checked variant (libdfsph_b200_checked.so) offers the same C ABI."""
    lib = _capi.load(_capi.CHECKED_LIB_PATH)
    for name in declared_symbols():
        assert hasattr(lib, name), name


def test_scene_defaults_match_reference_timestep(cuda_lib):
    s = _capi.DfsphScene()
    assert cuda_lib.dfsph_scene_defaults(C.byref(s)) == 0
    # SPH::TimeStep::TimeStep (TimeStep.cpp:23-44)
    assert s.max_iterations == 100 and s.max_iterations_v == 100
    assert s.max_error == pytest.approx(0.01) and s.max_error_v == pytest.approx(0.1)
    assert s.cfl_factor == pytest.approx(0.5) and s.cfl_max_time_step == pytest.approx(0.01)
    assert s.precision == 32 and s.neighbor_capacity >= 90


def test_struct_sizes_match_header(cuda_lib):
    assert C.sizeof(_capi.DfsphScene) % 8 == 0
    assert C.sizeof(_capi.DfsphStepStats) == 64
    assert C.sizeof(_capi.Surface) == 80


@pytest.mark.skipif(shutil.which("gcc") is None, reason="no C compiler")
def test_struct_layouts_match_c_compiler(tmp_path):
    """sizeof / offsetof of every struct of the header, from gcc, against the ctypes layouts."""
    structs = {"dfsph_scene": _capi.DfsphScene, "dfsph_step_stats": _capi.DfsphStepStats,
               "dfsph_surface": _capi.Surface}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "dfsph_c.h"', "int main(void) {"]
    for cname, cls in structs.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in cls._fields_:
            lines.append(f'printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines.append("return 0; }")
    src = tmp_path / "probe.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "probe"
    subprocess.run(["gcc", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {}
    for line in out:
        if line:
            a, b, c = line.split()
            got[(a, b)] = int(c)
    for cname, cls in structs.items():
        assert got[(cname, "size")] == C.sizeof(cls), cname
        for fname, _ in cls._fields_:
            assert got[(cname, fname)] == getattr(cls, fname).offset, (cname, fname)


def test_create_without_gpu_fails_loudly(cuda_lib):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    s = _capi.DfsphScene()
    cuda_lib.dfsph_scene_defaults(C.byref(s))
    ctx = C.c_void_p()
    code = cuda_lib.dfsph_create(C.byref(s), C.byref(ctx))
    assert code in (_capi.DFSPH_E_CUDA, _capi.DFSPH_E_NOMEM)
    assert not ctx.value
    assert cuda_lib.dfsph_last_error(None)


def test_invalid_arguments_rejected_before_cuda(cuda_lib):
    s = _capi.DfsphScene()
    cuda_lib.dfsph_scene_defaults(C.byref(s))
    s.precision = 16
    ctx = C.c_void_p()
    assert cuda_lib.dfsph_create(C.byref(s), C.byref(ctx)) == _capi.DFSPH_E_INVALID
    assert b"precision" in cuda_lib.dfsph_last_error(None)
    assert cuda_lib.dfsph_step(None, None) == _capi.DFSPH_E_INVALID
    assert cuda_lib.dfsph_destroy(None) == 0


@pytest.mark.parametrize("field,value,needle", [("neighbor_capacity", 0, "neighbor_capacity"),
                                                ("neighbor_capacity", 70000, "neighbor_capacity"),
                                                ("fluid_capacity", 0, "fluid_capacity"),
                                                ("particle_radius", 0.0, "particle_radius"),
                                                ("time_step", -1.0, "time_step")])
def test_create_rejects_bad_scene_before_touching_the_device(cuda_lib, field, value, needle):
    """Scene validation runs before any CUDA call: bad values give DFSPH_E_INVALID and a message
    naming the field, also on a machine without a GPU."""
    s = _capi.DfsphScene()
    cuda_lib.dfsph_scene_defaults(C.byref(s))
    setattr(s, field, value)
    ctx = C.c_void_p()
    assert cuda_lib.dfsph_create(C.byref(s), C.byref(ctx)) == _capi.DFSPH_E_INVALID
    assert not ctx.value
    assert needle in cuda_lib.dfsph_last_error(None).decode()
