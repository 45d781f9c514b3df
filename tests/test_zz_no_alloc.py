"""dslashCloverQcuNoAlloc: the clover hopping term for callers that cannot
allocate device memory (a framework whose caching allocator holds the memory
budget, a job under a hard device-memory cap, a latency-critical path).  It
must give the same result as dslashCloverQcu, which allocates its clover
scratch, call after call, and must reject lattices beyond its static scratch.

This file is collected last on purpose: if it fails, a run that stops at the
first failure has already run every other test."""
import numpy as np
import pytest

import oracle as O
from util import dev, empty_like_dev, host, rel

pytestmark = pytest.mark.gpu

# (lattice, gauge kind, seed, output parity): two different problems back to back
CASES = [([8, 8, 8, 8], "smooth", 31, 0), ([16, 8, 4, 8], "haar", 32, 1)]


def _inputs(latt, kind, seed):
    U = O.gauge_smooth(latt, 0.3, seed) if kind == "smooth" else O.gauge_haar(latt, seed)
    psi = O.fermion_gauss(O.half_shape(latt), seed + 1)
    return dev(U), dev(psi), U, psi


def _only_process_on_device():
    """True when NVML lists no compute process on the current GPU besides this one."""
    import os

    import torch

    try:
        import pynvml

        pynvml.nvmlInit()
        try:
            uuid = str(torch.cuda.get_device_properties(torch.cuda.current_device()).uuid)
            h = pynvml.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
            procs = pynvml.nvmlDeviceGetComputeRunningProcesses(h)
            return all(p.pid == os.getpid() for p in procs)
        finally:
            pynvml.nvmlShutdown()
    except Exception:
        return False


def test_no_alloc_matches_dslashCloverQcu_on_two_calls_in_a_row():
    import qcu_b200 as q

    for latt, kind, seed, parity in CASES:
        dU, dpsi, U, psi = _inputs(latt, kind, seed)
        out = empty_like_dev(O.half_shape(latt))
        rc = q.dslashCloverQcuNoAlloc(out, dpsi, dU, q.QcuParam(latt), parity)
        assert rc == 0, q.last_error()
        ref = empty_like_dev(O.half_shape(latt))
        q.dslashCloverQcu(ref, dpsi, dU, q.QcuParam(latt), parity)
        assert q.last_error()[0] == 0
        # the same kernels run in both: the results agree to the FP64 dslash bar
        assert rel(host(out), host(ref)) <= 1e-13
        assert np.isfinite(host(out)).all()
        # inputs are not modified
        assert np.array_equal(host(dU), U) and np.array_equal(host(dpsi), psi)


def test_no_alloc_allocates_nothing_and_rejects_oversize():
    import torch

    import qcu_b200 as q

    latt, kind, seed, parity = CASES[0]
    dU, dpsi, _, _ = _inputs(latt, kind, seed)
    out = empty_like_dev(O.half_shape(latt))
    assert q.dslashCloverQcuNoAlloc(out, dpsi, dU, q.QcuParam(latt), parity) == 0  # module loaded
    torch.cuda.synchronize()
    reserved_before = torch.cuda.memory_reserved()
    free_before = torch.cuda.mem_get_info()[0]
    assert q.dslashCloverQcuNoAlloc(out, dpsi, dU, q.QcuParam(latt), 1 - parity) == 0
    torch.cuda.synchronize()
    free_after = torch.cuda.mem_get_info()[0]
    assert torch.cuda.memory_reserved() == reserved_before  # nothing through torch's allocator
    # The free-memory figure is device-wide: another process on the GPU would
    # move it.  Exact equality is asserted only when this process is the only
    # one the driver lists on the device.
    if _only_process_on_device():
        assert free_after == free_before
    # beyond the static scratch: a clear error, nothing written
    big = [32, 32, 32, 32]
    assert O.vh(big) > q.noalloc_max_sites()
    poison = empty_like_dev((16,))
    rc = q.dslashCloverQcuNoAlloc(poison, poison, poison, q.QcuParam(big), 0)
    code, msg = q.last_error()
    assert rc != 0 and code == rc and "too large" in msg
    assert np.isnan(host(poison)).all()
