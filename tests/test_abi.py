"""CPU checks of the C-ABI boundary: the library loads, exports every entry point the header
declares, and the host-only entry points (rotation matrices, search grid, argument
validation) behave like the reference without touching a GPU."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    txt = open(os.path.join(ROOT, "include", "emc_b200.h")).read()
    return sorted(set(re.findall(r"EMC_API\s+[\w\s\*]+?\b(emc_\w+)\s*\(", txt)))


def test_header_declares_entry_points():
    names = header_functions()
    for must in ("emc_xform3d_create", "emc_xform3d_apply", "emc_xform3d_destroy", "emc_fft_plan", "emc_fft_r2c",
                 "emc_fft_c2r", "emc_fft_destroy", "emc_ctf2d", "emc_sf3d", "emc_search_run", "emc_cc_adjoint",
                 "emc_tsearch_run"):
        assert must in names


def test_library_exports_every_declared_symbol(built_lib):
    missing = [n for n in header_functions() if not hasattr(built_lib, n)]
    assert not missing, missing


def test_python_binding_covers_header(built_lib):
    from emclarity_b200 import _lib
    assert set(header_functions()) <= set(_lib.SIGNATURES)


def test_define_matrix_abi_matches_oracle(built_lib):
    from emclarity_b200 import api
    rng = np.random.default_rng(0)
    for _ in range(20):
        a = rng.uniform(-180, 180, 3)
        for d in ("forward", "inv"):
            assert np.abs(api.define_matrix(a, d) - O.define_matrix(a, d)).max() < 1e-14


@pytest.mark.parametrize("args", [("C1", 40, 10, 40, 10), ("C1", 180, 12, 48, 12), ("C1", 180, 15, 180, 15),
                                  ("C3", 60, 7.5, 90, 5), ("D2", 120, 10, 30, 10), ("O", 60, 10, 60, 10),
                                  ("I", 40, 8, 90, 9), ("I2", 40, 8, 90, 9), ("C1", -30, 10, 20, 5),
                                  ("C1", 0, 0, 0, 0), ("C1", 8, 2, 8, 2)])
def test_euler_search_abi_matches_oracle(built_lib, args):
    from emclarity_b200 import api
    g = api.euler_search(*args)
    g2 = O.euler_search_np(*args)
    assert g.shape == g2.shape
    assert np.abs(g - g2).max() < 1e-12


def test_euler_search_rejects_bad_symmetry(built_lib):
    from emclarity_b200 import _lib
    cnt = C.c_int(0)
    st = built_lib.emc_euler_search(b"X3", 10.0, 5.0, 10.0, 5.0, None, C.byref(cnt))
    assert st == _lib.EMC_E_ARG
    assert b"not recognised" in built_lib.emc_last_error()
    st = built_lib.emc_euler_search(b"C", 10.0, 5.0, 10.0, 5.0, None, C.byref(cnt))
    assert st == _lib.EMC_E_ARG


def test_null_arguments_are_rejected_before_any_device_work(built_lib):
    from emclarity_b200 import _lib
    assert built_lib.emc_xform3d_create(None, 4, 4, 4, 0, None, None) == _lib.EMC_E_ARG
    assert built_lib.emc_fft_plan(3, None, 1, None) == _lib.EMC_E_ARG
    dims = (C.c_int * 3)(100, 64, 64)  # 100 = 2^2 5^2 is not a compiled length
    h = C.c_void_p()
    assert built_lib.emc_fft_plan(3, dims, 1, C.byref(h)) == _lib.EMC_E_UNSUPPORTED
    assert built_lib.emc_search_run(None, None, 0, None, None, None, None) == _lib.EMC_E_ARG
    assert built_lib.emc_ctf2d(None, 8, 8, 1, 0, 0, None, None) == _lib.EMC_E_ARG
    assert built_lib.emc_sf3d(1, 1, None, None, None, None, None, None, None, None, 1, None, None, None, None,
                              None) == _lib.EMC_E_ARG
    # destroy functions accept NULL
    assert built_lib.emc_fft_destroy(None) == 0
    assert built_lib.emc_xform3d_destroy(None) == 0
    assert built_lib.emc_search_destroy(None) == 0


def test_batched_spectra_and_device_energy_search_reject_bad_arguments(built_lib):
    from emclarity_b200 import _lib
    fake = C.c_void_p(256)  # never dereferenced: every case below fails its argument checks first
    assert built_lib.emc_search_run_energies(None, None, 0, fake, None, None, None, None) == _lib.EMC_E_ARG
    assert built_lib.emc_particle_spectra(64, 0, fake, None, None, fake, fake, None) == _lib.EMC_E_ARG
    assert built_lib.emc_particle_spectra(64, 4, None, None, None, fake, fake, None) == _lib.EMC_E_ARG
    assert built_lib.emc_particle_spectra(100, 4, fake, None, None, fake, fake, None) == _lib.EMC_E_ARG
    assert b"not supported" in built_lib.emc_last_error()
    assert built_lib.emc_particle_spectra(64, 70000, fake, None, None, fake, fake, None) == _lib.EMC_E_ARG
    assert b"65535" in built_lib.emc_last_error()


def test_status_strings(built_lib):
    for s in (0, -1, -2, -3, -4, -5):
        assert built_lib.emc_status_string(s)
    assert b"sm_100a" in built_lib.emc_version()
