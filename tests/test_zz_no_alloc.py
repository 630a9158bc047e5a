"""The allocation-free metrics entry point against the regular one.

lfm_metrics_f64_noalloc serves callers that cannot call cudaMalloc (their
device memory is held by another allocator, or they must not allocate after
start-up) and so hold no library context: it keeps its per-CTA partials in a
static device array.  It must give the same metrics as lfm_metrics_f64, call
after call, since every call reuses that array.  This file is collected last
so that a run stopping at the first failure has run every other test.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# The two entry points reduce the same float64 terms over different CTA
# partitions, so sums agree to rounding; min/max and counts agree exactly.
REL_TOL = 1e-12
EXACT = ("chi_min", "chi_max", "well_fraction", "void_fraction", "interior_cells",
         "nonfinite_cells")


@pytest.fixture(scope="module")
def be(cuda_device):
    from lfm_b200 import B200Backend
    from lfm_b200.build import build_library

    build_library()
    return B200Backend(cuda_device)


def _noalloc(level, N, pr, prp, pi, pip, chi, dt=0.02, bf=0.3):
    import torch

    from lfm_b200 import _lib
    from lfm_b200.metrics import KEYS

    out = (ctypes.c_double * len(KEYS))()
    p = lambda t: None if t is None else t.data_ptr()  # noqa: E731
    _lib.call("lfm_metrics_f64_noalloc", level, p(pr), p(prp), p(pi), p(pip), p(chi), N, dt, 1.0,
              bf, 17.0, 18.0, out, torch.cuda.current_stream(chi.device).cuda_stream)
    return dict(zip(KEYS, (float(v) for v in out)))


def _check_same(got: dict, ref: dict) -> None:
    for k, v in ref.items():
        if k in EXACT:
            assert got[k] == v, k
        else:
            assert got[k] == pytest.approx(v, rel=REL_TOL, abs=1e-300), k


@pytest.mark.parametrize("level,N", [(0, 64), (1, 48), (2, 24)])
def test_noalloc_metrics_equal_regular_entry_point_twice(be, level, N):
    from lfm_b200.metrics import device_metrics

    rng = np.random.default_rng(10 + level)
    comps = 3 if level == 2 else 1
    shape = (comps * N**3,)
    pr, prp = (be.from_numpy(rng.standard_normal(shape).astype(np.float32)) for _ in range(2))
    pi, pip = ((be.from_numpy(rng.standard_normal(shape).astype(np.float32)) for _ in range(2))
               if level > 0 else (None, None))
    chi = be.from_numpy((18.5 + rng.standard_normal(N**3)).astype(np.float32))
    ref = device_metrics(be.context.handle, level, N, pr, prp, pi, pip, chi, 0.02, 1.0, 0.3)
    first = _noalloc(level, N, pr, prp, pi, pip, chi)
    second = _noalloc(level, N, pr, prp, pi, pip, chi)
    _check_same(first, ref)
    _check_same(second, ref)
    assert ref["interior_cells"] > 0 and ref["energy_total"] > 0


def test_noalloc_metrics_follow_new_inputs(be):
    """A call after a different lattice gives that lattice's metrics (no stale partials)."""
    from lfm_b200.metrics import device_metrics

    rng = np.random.default_rng(3)
    big = [be.from_numpy(rng.standard_normal(96**3).astype(np.float32)) for _ in range(3)]
    _noalloc(0, 96, big[0], big[1], None, None, big[2] + 19.0)
    small = [be.from_numpy(rng.standard_normal(16**3).astype(np.float32)) for _ in range(3)]
    chi = small[2] + 19.0
    ref = device_metrics(be.context.handle, 0, 16, small[0], small[1], None, None, chi, 0.02,
                         1.0, 0.3)
    _check_same(_noalloc(0, 16, small[0], small[1], None, None, chi), ref)


def test_noalloc_rejects_lattices_beyond_the_static_scratch(be):
    from lfm_b200._lib import LFM_ERR_CAPACITY, LfmError

    t = be.from_numpy(np.zeros(8, np.float32))  # never read: the size check comes first
    with pytest.raises(LfmError) as e:
        _noalloc(0, 600, t, t, None, None, t)
    assert e.value.code == LFM_ERR_CAPACITY
    assert "static scratch" in str(e.value)
