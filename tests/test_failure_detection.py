"""Failure detection without a GPU fault.

Every wait of the step kernels on an mbarrier is bounded by %globaltimer; when
it gives up, the kernel ORs LFM_ERR_DEVICE_TIMEOUT into a device status word
that the host reads with lfm_device_status, and returns.  The GPU test makes
such a wait run out on purpose (an mbarrier that nothing completes, waited on
through the kernels' own bounded wait) and checks the status word and that the
context still steps correctly afterwards.
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle import oracle as O


def test_selftest_rejects_limits_outside_range():
    from lfm_b200 import _lib
    from lfm_b200.build import build_library

    build_library()
    for bad in (0, 999, 2_000_000_000):
        with pytest.raises(_lib.LfmError) as e:
            _lib.call("lfm_selftest_device_timeout", bad, None)
        assert e.value.code == _lib.LFM_ERR_INVALID_ARG


@pytest.mark.gpu
def test_bounded_device_wait_gives_up_and_reports(cuda_device):
    from lfm_b200 import B200Backend, Evolver, _lib
    from lfm_b200.backend import _stream_handle
    from lfm_b200.config import gravity_only

    be = B200Backend(cuda_device)
    _lib.device_status(clear=True)
    _lib.call("lfm_selftest_device_timeout", 20_000_000, _stream_handle(be.device))  # 20 ms
    status = _lib.device_status(clear=True)
    assert status & _lib.LFM_ERR_DEVICE_TIMEOUT, status
    assert _lib.device_status() == 0

    # the context stays usable: resident steps still match the oracle bit for bit
    N = 16
    cfg = gravity_only(N)
    E = O.parity_seed_blob(N)
    ev = Evolver(cfg, backend=be)
    ev.set_psi_real(E)
    ev.evolve(5)
    lat = O.OracleLattice(cfg)
    lat.set_psi_real(E)
    lat.step(5)
    got = np.ascontiguousarray(ev.get_psi_real(), dtype=np.float32).ravel()
    assert np.array_equal(got.view(np.uint32), lat.pr.view(np.uint32))
    assert _lib.device_status() == 0


@pytest.mark.gpu
def test_reads_raise_after_a_device_wait_gave_up(cuda_device):
    """A timed-out wait is never silent: the next host read of the state raises."""
    from lfm_b200 import B200Backend, Evolver, _lib
    from lfm_b200.backend import _stream_handle
    from lfm_b200.config import gravity_only

    be = B200Backend(cuda_device)
    N = 16
    ev = Evolver(gravity_only(N), backend=be)
    ev.set_psi_real(O.parity_seed_blob(N))
    ev.evolve(2)
    ev.get_chi()  # nothing pending: reads normally
    _lib.call("lfm_selftest_device_timeout", 5_000_000, _stream_handle(be.device))  # 5 ms
    ev.evolve(1)
    with pytest.raises(_lib.LfmError) as e:
        ev.get_psi_real()
    assert e.value.code & _lib.LFM_ERR_DEVICE_TIMEOUT
    # the read cleared the word: later reads and synchronize() succeed
    ev.get_psi_real()
    ev.synchronize()
    _lib.call("lfm_selftest_device_timeout", 5_000_000, _stream_handle(be.device))
    with pytest.raises(_lib.LfmError):
        be.synchronize()
    assert _lib.device_status() == 0
