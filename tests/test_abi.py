"""The C-ABI libraries load and export every function their headers declare;
argument validation happens before any device work (CPU only)."""
import ctypes as C
import os
import re
import subprocess

import pytest

from ucns3d_b200 import _native as N
from ucns3d_b200 import build
from ucns3d_b200.config import make_config
from ucns3d_b200.mesh import SCHEME_MUSCL, Mesh

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared(header):
    txt = open(os.path.join(ROOT, "include", header)).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(uc[gp]_[a-z0-9_]+)\s*\(", txt)))


def _exported(lib):
    out = subprocess.run(["nm", "-D", "--defined-only", lib], capture_output=True, text=True, check=True).stdout
    return {ln.split()[-1] for ln in out.splitlines() if " T " in ln}


@pytest.fixture(scope="module")
def engine_lib():
    return build.build_engine()


def test_engine_exports_header(engine_lib):
    decl = _declared("ucns3d_gpu.h")
    assert len(decl) >= 20
    missing = set(decl) - _exported(engine_lib)
    assert not missing, missing
    assert set(N.ENGINE_SYMBOLS) <= set(decl)


def test_prep_exports_header():
    lib = build.build_prep()
    decl = _declared("ucns3d_prep.h")
    missing = set(decl) - _exported(lib)
    assert not missing, missing


def test_build_targets_sm100a():
    assert build.GENCODE == ["-gencode", "arch=compute_100a,code=sm_100a"]


def test_create_validates_before_device(engine_lib):
    lib = N.engine()
    m = Mesh.box_hex(4, 4, 4).prepare(SCHEME_MUSCL, 1)
    cfg = make_config(m)
    bad = N.UcgConfig.from_buffer_copy(cfg)
    bad.ideg = 7  # inconsistent with iorder 1
    h = C.c_void_p()
    assert lib.ucg_create(C.byref(bad), m.ncells, 0, C.byref(h)) == N.UCG_EINVAL
    assert b"inconsistent" in lib.ucg_create_error()
    assert lib.ucg_create(C.byref(cfg), 0, 0, C.byref(h)) == N.UCG_EINVAL


def test_create_rejects_unsupported_codes(engine_lib):
    """Riemann solvers 1-5 and 9, limiters 1-9 and characteristic WENO (WENO
    only) are accepted; anything else is refused before any device work."""
    lib = N.engine()
    m = Mesh.box_hex(4, 4, 4).prepare(SCHEME_MUSCL, 1)
    cfg = make_config(m)
    h = C.c_void_p()
    for field, value in (("riemann", 6), ("riemann", 0), ("limiter", 10), ("limiter", 0), ("wenwrt", 2),
                         ("wenwrt", 3)):
        bad = N.UcgConfig.from_buffer_copy(cfg)
        setattr(bad, field, value)
        assert lib.ucg_create(C.byref(bad), m.ncells, 0, C.byref(h)) == N.UCG_EINVAL, (field, value)
        assert not h.value


def test_create_without_gpu_reports_cuda_error(engine_lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    lib = N.engine()
    m = Mesh.box_hex(4, 4, 4).prepare(SCHEME_MUSCL, 1)
    cfg = make_config(m)
    h = C.c_void_p()
    assert lib.ucg_create(C.byref(cfg), m.ncells, 0, C.byref(h)) == N.UCG_ECUDA
    assert not h.value
