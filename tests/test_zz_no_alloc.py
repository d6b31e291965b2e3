"""tg_corner_spectra_noalloc: the allocation-free entry point for callers that
must not allocate device memory (fixed memory budgets, caller-owned device
pools, checks slotted between other GPU work).

It must give the same corner spectra as tg_corner_spectrum, which allocates
its scratch on the fly, on two calls in a row (the static scratch keeps the
previous call's contents).  This file is collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

from tenes_b200 import _lib
from tests._helpers import gpu_env, make_lattice, random_tensors

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("is_complex", [False, True])
def test_noalloc_spectra_match_allocating_path(is_complex):
    import torch

    lat = make_lattice(2, 2, 2)
    chi = 12
    lib = _lib.load()
    for call in range(2):  # two calls in a row through the same static table
        Tn = random_tensors(lat, 100 + call, is_complex)
        env = gpu_env(lat, Tn, chi, is_complex, max_ctm_iteration=2)
        env.calc_ctm_environment(True)
        dt = torch.complex128 if is_complex else torch.float64
        mats = [torch.from_numpy(env.get_env(w, i)).to(device="cuda:0", dtype=dt).contiguous()
                for i in range(lat.N_UNIT) for w in range(4)]
        ptrs = (C.c_void_p * len(mats))(*[m.data_ptr() for m in mats])
        out = torch.full((len(mats), chi), -1.0, dtype=torch.float64, device="cuda:0")
        torch.cuda.synchronize()
        code = lib.tg_corner_spectra_noalloc(ptrs, len(mats), chi, int(is_complex),
                                             C.cast(out.data_ptr(), C.POINTER(C.c_double)), None)
        assert code == _lib.TG_OK, lib.tg_last_error().decode()
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        for b, (i, w) in enumerate([(i, w) for i in range(lat.N_UNIT) for w in range(4)]):
            ref = env.corner_spectrum(w, i)
            np.testing.assert_allclose(got[b], ref, rtol=1e-12, atol=1e-14)
        env.close()


def test_noalloc_rejects_oversized_requests():
    lib = _lib.load()
    ptrs = (C.c_void_p * 1)(1)
    out = C.c_double()
    assert lib.tg_corner_spectra_noalloc(ptrs, 1025, 8, 0, C.byref(out), None) == _lib.TG_E_INPUT
    assert "1024" in lib.tg_last_error().decode()
    assert lib.tg_corner_spectra_noalloc(ptrs, 1, 161, 0, C.byref(out), None) == _lib.TG_E_INPUT
    assert lib.tg_corner_spectra_noalloc(ptrs, 1, 113, 1, C.byref(out), None) == _lib.TG_E_INPUT
