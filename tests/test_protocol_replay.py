"""The reference Evolver's own call sequence, replayed against B200Backend.

tests/golden/make_protocol_trace.py ran the reference's ``Evolver``
(lfm/core/evolver.py) on its CPU backend and logged, in order, every call it
made to the backend and every operation on the arrays the backend gave it:
``from_numpy``, ``create_boundary_mask``, the ``step_*`` calls with their
A/B buffers, the setters' ``buf[:] = data``, freeze_chi's ``.copy()``
snapshots and restores, and each ``to_numpy`` read with the value it returned.
Here that log drives ``B200Backend`` on the GPU step by step, so the
reference Evolver's exact use of the backend protocol
(lfm/core/backends/protocol.py:17-144) runs through the B200 path, and every
read must equal the reference's: bit for bit at REAL and COMPLEX and at COLOR
without S_a; within the stated S_a tolerance where cuFFT enters.
"""

from __future__ import annotations

import json

import numpy as np
import pytest

from conftest import load_golden

# COLOR with the S_a solve: cuFFT's float32 transforms against NumPy's
# (complex64 forward, float64 inverse), per read, max-relative
SA_RTOL = 1e-5


def _trace():
    g = load_golden("protocol_trace.npz")
    return g, json.loads(str(g["trace"]))


def test_trace_covers_the_protocol():
    """The recorded sessions use every backend entry point and array operation."""
    _, t = _trace()
    ops = {o["op"] for o in t["ops"]}
    assert {"new", "mask", "copy", "assign", "to_numpy", "step_real", "step_complex",
            "step_color"} <= ops
    assert [s["tag"] for s in t["sessions"]] == ["real", "complex", "color"]


def replay(be, g, ops):
    """Run the logged operations on `be`; returns [(recorded key, value read)]."""
    H = {}
    reads = []

    def arg(a):
        return H[a["h"]] if "h" in a else a["v"]

    for o in ops:
        op = o["op"]
        if op == "new":
            H[o["out"]] = be.from_numpy(g[o["data"]])
        elif op == "mask":
            H[o["out"]] = be.create_boundary_mask(o["N"], o["boundary_fraction"])
        elif op == "copy":
            H[o["out"]] = H[o["src"]].copy()
        elif op == "assign":
            H[o["dst"]][:] = arg(o["src"])
        elif op == "to_numpy":
            reads.append((o["result"], be.to_numpy(H[o["src"]])))
        else:
            getattr(be, op)(*[arg(a) for a in o["args"]],
                            **{k: arg(v) for k, v in o["kwargs"].items()})
    return reads


@pytest.mark.gpu
@pytest.mark.parametrize("tag", ["real", "complex", "color"])
def test_reference_evolver_calls_replayed_on_b200(cuda_device, tag):
    from lfm_b200 import B200Backend, _lib

    g, t = _trace()
    s = next(x for x in t["sessions"] if x["tag"] == tag)
    be = B200Backend(cuda_device)
    reads = replay(be, g, t["ops"][s["first"]:s["last"]])
    assert len(reads) > 0
    for key, got in reads:
        want = g[key]
        assert got.shape == want.shape and got.dtype == np.float32, key
        if tag == "color":
            err = np.abs(got.astype(np.float64) - want).max() / max(np.abs(want).max(), 1e-30)
            assert err <= SA_RTOL, (key, err)
        else:
            assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), key
    assert _lib.device_status() == 0


class _OracleArrays:
    """The oracle behind the same protocol, with NumPy arrays (CPU check of the log)."""

    def __init__(self):
        from oracle import oracle as O

        self._O = O
        self._be = O.OracleBackend()

    def from_numpy(self, a):
        return np.array(a, dtype=np.float32, copy=True)

    def create_boundary_mask(self, N, boundary_fraction):
        return self._O.boundary_mask(N, boundary_fraction)

    def to_numpy(self, a):
        return np.array(a, copy=True)

    def __getattr__(self, name):
        return getattr(self._be, name)


@pytest.mark.parametrize("tag", ["real", "complex", "color"])
def test_trace_replays_bit_exact_on_the_oracle(tag):
    """The log is complete: replayed on the oracle, every read equals the reference's."""
    g, t = _trace()
    s = next(x for x in t["sessions"] if x["tag"] == tag)
    reads = replay(_OracleArrays(), g, t["ops"][s["first"]:s["last"]])
    assert len(reads) > 0
    for key, got in reads:
        assert np.array_equal(got.view(np.uint32), g[key].view(np.uint32)), key
