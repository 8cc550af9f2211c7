"""The allocation-free single-particle search (emc_search_plain_noalloc).

It exists for callers that may not allocate device memory while they run -- hosts whose own
memory pool owns the GPU (MATLAB's gpuArray allocator, a framework caching allocator) and
loops that must not allocate after start-up.  Its output must equal the regular entry point's
on the same inputs, call after call, although every call reuses the same static scratch.
This file is collected last so that a failure here leaves every other test already run."""
import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _noalloc(lib, ref, mask, n, q, e, prior, grid, radius, interp, cc, pk, best):
    ptp = np.ascontiguousarray(grid, dtype=np.float64)
    pr = np.ascontiguousarray(np.asarray(prior).flatten(order="F"))
    sh = (C.c_float * 3)(0, 0, 0)
    return lib.emc_search_plain_noalloc(
        C.c_void_p(ref.data_ptr()), C.c_void_p(mask.data_ptr()), n, C.c_void_p(q.data_ptr()), e,
        pr.ctypes.data_as(C.POINTER(C.c_double)), sh, ptp.ctypes.data_as(C.POINTER(C.c_double)), len(grid), radius,
        interp, C.c_void_p(cc.data_ptr()), C.c_void_p(pk.data_ptr()), C.c_void_p(best.data_ptr()),
        C.c_void_p(torch.cuda.current_stream().cuda_stream))


# (box, interpolation, peak radius, orientations): every box, the three interpolation modes, and the
# tightest scratch layout -- 128^3 at radius 15, two evaluations per chunk -- over several chunks
CASES = [(64, 0, 7, 0), (64, 1, 5, 60), (96, 2, 9, 40), (128, 0, 15, 9), (128, 1, 15, 7)]


@pytest.mark.parametrize("n,interp,radius,n_orient", CASES)
def test_noalloc_matches_search_run_twice(built_lib, cuda, n, interp, radius, n_orient):
    from emclarity_b200 import _lib as L
    from emclarity_b200 import api, synthetic
    case = synthetic.PlainCase(seed=9, n=n)
    g = case.to_gpu()
    grid = case.grid if not n_orient else case.grid[:: max(1, len(case.grid) // n_orient)][:n_orient]
    q, e = api.particle_spectrum(g["particle"], g["weight"])
    prior = api.define_matrix([15.0, 30.0, -20.0], "inv")
    s = api.Search(peak_radius=radius, interp={0: "linear", 1: "cubic", 2: "linear_border"}[interp])
    rid = s.add_reference(g["ref"], g["mask"])
    s.set_orientations(grid)
    cc_ref, pk_ref, best_ref = s.run_host([s.particle(q, e.item(), rid, prior=prior, orient_count=len(grid))])
    s.close()

    lib = L.load()
    n_or = len(grid)
    free = []
    for _ in range(2):
        cc = torch.full((n_or,), float("nan"), device="cuda")
        pk = torch.full((n_or, 3), -99, dtype=torch.int32, device="cuda")
        best = torch.zeros((1, 5), dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        free.append(torch.cuda.mem_get_info()[0])
        st = _noalloc(lib, g["ref"], g["mask"], n, q, e.item(), prior, grid, radius, interp, cc, pk, best)
        assert st == 0, lib.emc_last_error()
        torch.cuda.synchronize()
        free.append(torch.cuda.mem_get_info()[0])
        ccn, pkn, bn = cc.cpu().numpy(), pk.cpu().numpy(), best.cpu().numpy()[0]
        assert np.allclose(ccn, cc_ref, rtol=1e-4, atol=1e-6)
        assert np.array_equal(pkn, pk_ref)
        assert bn[1] == best_ref[0][1] and tuple(bn[2:]) == tuple(best_ref[0][2])
        assert abs(np.frombuffer(np.int32(bn[0]).tobytes(), np.float32)[0] - best_ref[0][0]) <= 1e-4 * abs(
            best_ref[0][0])
    # the second call (the device already set up) allocates no device memory
    assert free[3] == free[2], (free[2], free[3])


def test_noalloc_rejects_sizes_beyond_its_scratch(built_lib, cuda):
    from emclarity_b200 import _lib as L
    lib = L.load()
    x = torch.zeros(8, device="cuda")
    eye = np.ascontiguousarray(np.eye(3).flatten())
    ptp = np.zeros((5000, 3))
    args = lambda n, no, r: (C.c_void_p(x.data_ptr()), None, n, C.c_void_p(x.data_ptr()), 1.0,  # noqa: E731
                              eye.ctypes.data_as(C.POINTER(C.c_double)), None,
                              ptp.ctypes.data_as(C.POINTER(C.c_double)), no, r, 0, None, None, None, None)
    assert lib.emc_search_plain_noalloc(*args(64, 5000, 7)) == L.EMC_E_ARG
    assert b"at most 4096" in lib.emc_last_error()
    assert lib.emc_search_plain_noalloc(*args(256, 10, 7)) == L.EMC_E_ARG
    assert lib.emc_search_plain_noalloc(*args(64, 10, 40)) == L.EMC_E_ARG
