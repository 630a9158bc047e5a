"""Record how the reference's own Evolver drives its backend; write protocol_trace.npz.

Run in a checkout that has the reference package importable::

    PYTHONPATH=<reference checkout> PYTHONDONTWRITEBYTECODE=1 python tests/golden/make_protocol_trace.py

The reference's ``Evolver`` (lfm/core/evolver.py) runs scripted sessions on
its CPU backend (``NumpyBackend``, lfm/core/backends/numpy_backend.py) wrapped
in a recorder.  Every interaction of the Evolver with the backend and with the
arrays the backend handed out is logged in order:

* ``new``      -- ``from_numpy(host)``: the host array is stored in the file;
* ``mask``     -- ``create_boundary_mask(N, boundary_fraction)``;
* ``copy``     -- ``array.copy()`` (the freeze_chi snapshot, evolver.py:160-166);
* ``assign``   -- ``buf[:] = data`` or ``np.copyto(buf, data)`` (the setters);
* ``step_real`` / ``step_complex`` / ``step_color`` -- the call with its
  positional and keyword arguments (arrays by handle, scalars by value);
* ``to_numpy`` -- a read; the value the reference backend returned is stored.

tests/test_protocol_replay.py replays the log against ``B200Backend`` on the
GPU, so the reference Evolver's exact call sequence (A/B toggling, the setters'
slice assignments, freeze_chi's copies and restores, callback reads) is driven
through the B200 backend, and every read is compared with the reference's.
"""

from __future__ import annotations

import json
from pathlib import Path

import numpy as np

import lfm.core.evolver as evolver_module
from lfm.config import FieldLevel, SimulationConfig
from lfm.core.backends.numpy_backend import NumpyBackend
from lfm.core.evolver import Evolver

OUT = Path(__file__).resolve().parent / "protocol_trace.npz"
LAMBDA_H = 4.0 / 31.0
CC = dict(kappa_c=1.0 / 189.0, epsilon_cc=2.0 / 17.0, kappa_string=1.0 / 189.0)


class Recorder:
    def __init__(self):
        self.ops: list = []
        self.data: dict = {}
        self.inside = 0  # > 0 while the wrapped backend computes (not logged)
        self.next_handle = 0

    def handle(self, arr) -> int:
        h = self.next_handle
        self.next_handle += 1
        arr._h = h
        return h

    def store(self, prefix: str, a: np.ndarray) -> str:
        key = f"{prefix}{len(self.data)}"
        self.data[key] = np.array(a, copy=True)
        return key


REC = Recorder()


class Traced(np.ndarray):
    """A backend array that logs what the Evolver does with it."""

    _h = -1

    def __array_finalize__(self, obj):
        self._h = -1  # results of arithmetic are anonymous

    def copy(self, *args, **kwargs):
        out = np.ndarray.copy(self, *args, **kwargs).view(Traced)
        if REC.inside == 0 and self._h >= 0:
            REC.ops.append({"op": "copy", "src": self._h, "out": REC.handle(out)})
        return out

    def __setitem__(self, key, value):
        if REC.inside == 0 and self._h >= 0:
            if not (isinstance(key, slice) and key == slice(None)):
                raise NotImplementedError(f"partial assignment {key!r} not traced")
            REC.ops.append({"op": "assign", "dst": self._h, "src": _ref(value)})
        np.ndarray.__setitem__(self.view(np.ndarray), key, np.asarray(value))

    def __array_function__(self, func, types, args, kwargs):
        if func is np.copyto and REC.inside == 0 and getattr(args[0], "_h", -1) >= 0:
            REC.ops.append({"op": "assign", "dst": args[0]._h, "src": _ref(args[1])})
            np.copyto(args[0].view(np.ndarray), np.asarray(args[1]))
            return None
        return super().__array_function__(func, types, args, kwargs)


def _ref(v):
    h = getattr(v, "_h", -1)
    if h >= 0:
        return {"h": h}
    raise NotImplementedError("assignment from an array the backend did not hand out")


def _arg(v):
    if isinstance(v, Traced) and v._h >= 0:
        return {"h": v._h}
    if v is None or isinstance(v, (bool, int, float)):
        return {"v": v}
    raise TypeError(f"untraceable argument {type(v).__name__}")


class RecordingBackend:
    """NumpyBackend with every Evolver-visible interaction logged."""

    def __init__(self):
        self.inner = NumpyBackend()

    @property
    def name(self):
        return self.inner.name

    def from_numpy(self, arr):
        out = np.array(arr, dtype=np.float32, copy=True).view(Traced)
        REC.ops.append({"op": "new", "out": REC.handle(out), "data": REC.store("d", arr)})
        return out

    def create_boundary_mask(self, N, boundary_fraction):
        out = np.asarray(self.inner.create_boundary_mask(N, boundary_fraction)).view(Traced)
        REC.ops.append({"op": "mask", "out": REC.handle(out), "N": int(N),
                        "boundary_fraction": float(boundary_fraction)})
        return out

    def to_numpy(self, arr):
        out = np.array(np.asarray(arr), dtype=np.float32, copy=True)
        REC.ops.append({"op": "to_numpy", "src": arr._h, "result": REC.store("r", out)})
        return out

    def synchronize(self):
        pass

    def _step(self, name, args, kwargs):
        REC.ops.append({"op": name, "args": [_arg(a) for a in args],
                        "kwargs": {k: _arg(v) for k, v in kwargs.items()}})
        REC.inside += 1
        try:
            plain = [a.view(np.ndarray) if isinstance(a, Traced) else a for a in args]
            kw = {k: (v.view(np.ndarray) if isinstance(v, Traced) else v)
                  for k, v in kwargs.items()}
            getattr(self.inner, name)(*plain, **kw)
        finally:
            REC.inside -= 1

    def step_real(self, *args, **kwargs):
        self._step("step_real", args, kwargs)

    def step_complex(self, *args, **kwargs):
        self._step("step_complex", args, kwargs)

    def step_color(self, *args, **kwargs):
        self._step("step_color", args, kwargs)


def blob(N, centre, amp, sigma):
    x = np.arange(N, dtype=np.float64)
    d2 = sum(((x - c) ** 2).reshape([-1 if i == a else 1 for i in range(3)])
             for a, c in enumerate(centre))
    return (amp * np.exp(-d2 / (2.0 * sigma * sigma))).astype(np.float32)


def session(tag: str, cfg: SimulationConfig, script) -> dict:
    first = len(REC.ops)
    ev = Evolver(cfg, backend="cpu")
    script(ev)
    return {"tag": tag, "first": first, "last": len(REC.ops),
            "config": {k: (int(v) if isinstance(v, FieldLevel) else v)
                       for k, v in vars(cfg).items()
                       if isinstance(v, (int, float, bool, FieldLevel))}}


def main():
    evolver_module.get_backend = lambda preference="auto": RecordingBackend()
    rng = np.random.default_rng(11)
    N = 16
    E = blob(N, (7.5, 8.0, 8.5), 1.5, 2.0)
    sessions = []

    def cb(ev, step):
        ev.get_chi()

    def real_script(ev):
        ev.set_psi_real(E)
        ev.evolve(7)
        ev.get_psi_real(), ev.get_chi()
        ev.set_psi_real_prev(ev.get_psi_real() * np.float32(0.999))
        ev.evolve(3, freeze_chi=True)
        ev.get_psi_real(), ev.get_chi(), ev.get_psi_real_prev()
        ev.set_psi_real_current(ev.get_psi_real() + np.float32(1e-3))
        ev.evolve(4, callback=cb)
        ev.get_psi_real(), ev.get_chi(), ev.get_psi_real_prev()

    sessions.append(session("real", SimulationConfig(grid_size=N, boundary_fraction=0.2,
                                                     report_interval=2), real_script))

    def complex_script(ev):
        ev.set_psi_real(E)
        ev.set_psi_imag(0.5 * E)
        ev.set_chi((19.0 + 1e-2 * rng.standard_normal((N,) * 3)).astype(np.float32))
        ev.evolve(5)
        ev.set_chi_current(ev.get_chi() - np.float32(1e-3))
        ev.set_chi_prev(ev.get_chi())
        ev.evolve(4, freeze_chi=True)
        ev.set_psi_imag_prev(ev.get_psi_imag())
        ev.set_psi_imag_current(ev.get_psi_imag() * np.float32(1.01))
        ev.evolve(6)
        ev.get_psi_real(), ev.get_psi_imag(), ev.get_chi(), ev.get_psi_imag_prev()

    sessions.append(session("complex", SimulationConfig(grid_size=N, boundary_fraction=0.2,
                                                        field_level=FieldLevel.COMPLEX,
                                                        lambda_self=LAMBDA_H), complex_script))

    def color_script(ev):
        pr = np.stack([E, 0.5 * E, -0.25 * E])
        ev.set_psi_real(pr)
        ev.set_psi_imag(np.stack([0.3 * E, -0.2 * E, 0.1 * E]))
        ev.evolve(6)
        ev.get_psi_real(), ev.get_psi_imag(), ev.get_chi(), ev.get_sa_fields()
        ev.evolve(3, freeze_chi=True)
        ev.get_psi_real(), ev.get_chi()

    sessions.append(session("color", SimulationConfig(grid_size=N, boundary_fraction=0.2,
                                                      field_level=FieldLevel.COLOR,
                                                      lambda_self=LAMBDA_H,
                                                      kappa_tube=30.0 / 63.0, **CC),
                            color_script))

    np.savez_compressed(OUT, trace=json.dumps({"ops": REC.ops, "sessions": sessions}),
                        **REC.data)
    print(f"wrote {OUT}: {len(REC.ops)} operations, {len(REC.data)} arrays")


if __name__ == "__main__":
    main()
