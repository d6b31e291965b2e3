"""C-ABI checks that need no GPU: the library loads, exports every symbol
declared in include/tenes_gpu.h, and rejects bad input before touching CUDA."""
import ctypes as C
import os
import re

import pytest

from tenes_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    txt = open(os.path.join(ROOT, "include", "tenes_gpu.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b((?:tg|tenes_gpu)_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    names = declared_symbols()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(_lib.EXPORTED)


def test_params_default_matches_reference():
    lib = _lib.load()
    p = _lib.Params()
    lib.tg_params_default(C.byref(p))
    # PEPS_Parameters.cpp:30-77
    assert p.chi == 2 and p.max_ctm_iteration == 100
    assert p.inverse_projector_cut == 1e-12 and p.ctm_convergence_epsilon == 1e-6
    assert p.projector_corner == 1 and p.use_rsvd == 0 and p.rsvd_oversampling_factor == 2.0
    assert p.inverse_lambda_cut == 1e-12
    assert p.mixed == 0 and p.cuda_graph == 1
    assert lib.tg_version().decode().startswith("tenes_gpu")


def _create(LX, LY, pd, vd, chi=4):
    lib = _lib.load()
    p = _lib.Params()
    lib.tg_params_default(C.byref(p))
    p.chi = chi
    pdc = (C.c_int * len(pd))(*pd)
    vdc = (C.c_int * (4 * len(vd)))(*[x for v in vd for x in v])
    desc = _lib.LatticeDesc(LX, LY, 0, pdc, vdc)
    h = C.c_void_p()
    return lib.tg_ctx_create(C.byref(desc), C.byref(p), 0, 0, C.byref(h)), h


def test_bad_lattice_is_input_error():
    code, h = _create(2, 2, [2] * 4, [[2, 2, 2, 2], [3, 2, 2, 2], [2, 2, 2, 2], [2, 2, 2, 2]])
    assert code == _lib.TG_E_INPUT
    assert "mismatch" in _lib.load().tg_last_error().decode()
    assert not h.value
    code, h = _create(0, 2, [2] * 4, [[2] * 4] * 4)
    assert code == _lib.TG_E_INPUT


def test_null_context_is_state_error():
    lib = _lib.load()
    assert lib.tg_ctm_init(None) == _lib.TG_E_STATE
    assert lib.tg_ctx_destroy(None) == _lib.TG_OK
