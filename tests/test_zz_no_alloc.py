"""sbr_run_noalloc: the sweep entry point that allocates no device memory.

It exists for callers that cannot call cudaMalloc while they run -- code that
works inside a fixed device-memory budget owned by a pool, or whose other streams
must not be stalled by the synchronisation cudaMalloc / cudaFree perform.  Its
scratch lives in a fixed-size device array inside libsbr; the caller owns the
output arrays (here two torch tensors, allocated by the test, not by the call).

The test calls it twice in a row through the C ABI and checks both results
against the allocating entry point sbr_run, with the tolerance of the other GPU
tests for identical arithmetic (the two paths build the same tables and run the
same kernels, so the fields agree to rounding of the final conversion), and that
the device's free memory is the same before and after the second call.  It also
checks the size limit.  This file sorts last so a failure here stops a `-x` run
only after every other test has run; it passes alone as well.
"""
import ctypes as C

import numpy as np
import pytest

import sagittasbr_b200 as sbr
from sagittasbr_b200 import _lib
from sagittasbr_b200 import meshes as M

pytestmark = pytest.mark.gpu


def _call(scene, job_c, field, stats, opts):
    return _lib.lib().sbr_run_noalloc(scene.handle, C.byref(job_c), C.c_void_p(field.data_ptr()),
                                      C.c_void_p(stats.data_ptr()) if stats is not None else None, C.byref(opts))


def test_noalloc_matches_allocating_run_on_two_calls():
    import torch
    assert torch.cuda.is_available(), "GPU test"
    v, t = M.icosphere(3, 1.0)
    th = np.full(40, 90.0)
    ph = np.linspace(0.0, 351.0, 40)
    fr = [1.5e9, 3e9]
    job = sbr.JobSpec(th, ph, fr, 64, 64, 2.0, 3)
    with sbr.Scene(v, t, device=0) as scene:
        ref = sbr.run(scene, job)
        job_c = job.to_c()
        opts = _lib.RunOpts()  # batched, mixed precision, scene stream
        field = torch.full((2 * len(th) * len(fr),), -1.0, dtype=torch.float64, device="cuda")
        stats = torch.full((4 * len(th),), -1, dtype=torch.int64, device="cuda")
        torch.cuda.synchronize()
        free_before = None
        for call in range(2):
            if call == 1:
                # the first call may load the module; from then on nothing is allocated
                torch.cuda.synchronize()
                free_before = torch.cuda.mem_get_info()[0]
            _lib.check(_call(scene, job_c, field, stats, opts), "sbr_run_noalloc")
            if call == 1:
                assert torch.cuda.mem_get_info()[0] == free_before, "device memory changed across the call"
            f = field.cpu().numpy()
            got = f[0::2] + 1j * f[1::2]
            np.testing.assert_allclose(got, ref.field, rtol=1e-12, atol=1e-14 * np.abs(ref.field).max())
            np.testing.assert_array_equal(stats.cpu().numpy().view(np.uint64).reshape(len(th), 4), ref.stats)
            field.fill_(-1.0)
            torch.cuda.synchronize()


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch
    v, t = M.box(1.0)
    with sbr.Scene(v, t, device=0) as scene:
        opts = _lib.RunOpts()
        field = torch.zeros(2 * 2048, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        too_many = sbr.JobSpec(np.zeros(2048), np.zeros(2048), [1e9], 8, 8, 2.0, 2).to_c()
        assert _call(scene, too_many, field, None, opts) == 5  # SBR_ERR_TOO_LARGE
        assert b"SBR_NOALLOC_MAX_ANGLES" in _lib.lib().sbr_last_error()
        too_many_samples = sbr.JobSpec(np.zeros(64), np.zeros(64), np.linspace(1e9, 2e9, 65), 8, 8, 2.0, 2).to_c()
        assert _call(scene, too_many_samples, field, None, opts) == 5
