"""Checkpoints in the reference's npz format, with an exact resume.

The reference (lfm/simulation.py:1474-1565, wrapped by lfm/io/__init__.py)
stores the current Psi and chi, S_a, a host snapshot of Psi used for the
kinetic energy, the config and the metric history as JSON.  On load it sets
each field with set_psi_real / set_chi, which makes the previous step equal
to the current one: the leapfrog velocity is lost and the resumed run leaves
the uninterrupted one.

``save_checkpoint`` writes the same keys, so the reference can read the file,
plus the leapfrog previous fields as the step reads them
(``leapfrog_psi_real_prev``, ``leapfrog_psi_imag_prev``,
``leapfrog_chi_prev``).  ``load_checkpoint`` restores them when present, so
a resumed run is bit-identical to an uninterrupted one; a file the reference
wrote loads with the reference's semantics.
"""

from __future__ import annotations

import json
from pathlib import Path

import numpy as np

from .config import BoundaryType, FieldLevel, SimulationConfig

EXACT_KEYS = ("leapfrog_psi_real_prev", "leapfrog_psi_imag_prev", "leapfrog_chi_prev")


def config_to_json(config) -> str:
    d = {k: v for k, v in vars(config).items() if not k.startswith("_")}
    for k, v in d.items():
        if hasattr(v, "value"):
            d[k] = v.value
    return json.dumps(d)


def config_from_json(text: str) -> SimulationConfig:
    d = json.loads(text)
    d["field_level"] = FieldLevel(d["field_level"])
    d["boundary_type"] = BoundaryType(d["boundary_type"])
    for key in ("dx", "sigma"):  # derived in __post_init__
        d.pop(key, None)
    return SimulationConfig(**d)


def save_checkpoint(evolver, path, history=None, psi_snapshot=None) -> None:
    """Write the evolver's state to an npz file.

    history: the metric history list to store (JSON); psi_snapshot: the
    (psi_r, psi_i) host snapshot a Simulation keeps for its kinetic energy,
    stored as psi_real_prev / psi_imag_prev as the reference does.
    """
    path = Path(path)
    path.parent.mkdir(parents=True, exist_ok=True)
    data: dict[str, object] = {
        "step": np.int64(evolver.step),
        "chi": evolver.get_chi(),
        "psi_real": evolver.get_psi_real(),
    }
    pi = evolver.get_psi_imag()
    if pi is not None:
        data["psi_imag"] = pi
    if psi_snapshot is not None:
        data["psi_real_prev"] = np.asarray(psi_snapshot[0], np.float32)
        if psi_snapshot[1] is not None:
            data["psi_imag_prev"] = np.asarray(psi_snapshot[1], np.float32)
    sa = evolver.get_sa_fields() if hasattr(evolver, "get_sa_fields") else None
    if sa is not None:
        data["sa_fields"] = sa
    data["config_json"] = np.array(config_to_json(evolver.config))
    data["history_json"] = np.array(json.dumps(history or []))
    # the previous fields the next step reads: what makes the resume exact
    data["leapfrog_psi_real_prev"] = evolver.get_psi_real_prev()
    if pi is not None:
        data["leapfrog_psi_imag_prev"] = evolver.get_psi_imag_prev()
    data["leapfrog_chi_prev"] = evolver.get_chi_prev()
    np.savez_compressed(str(path), **data)


def read_checkpoint(path) -> dict:
    """The file's contents on the host: config, step, fields, history (no device)."""
    with np.load(str(path), allow_pickle=False) as z:
        out = {k: z[k] for k in z.files}
    out["config"] = config_from_json(str(out.pop("config_json")))
    out["history"] = json.loads(str(out.pop("history_json"))) if "history_json" in out else []
    out["step"] = int(out["step"])
    out["exact"] = all(k in out for k in ("leapfrog_psi_real_prev", "leapfrog_chi_prev"))
    return out


def load_checkpoint(path, backend="auto", buffers: str = "resident"):
    """An Evolver restored from a checkpoint; returns (evolver, contents).

    With the leapfrog previous fields in the file the next step is the one the
    saved run would have taken; without them (a reference file) the previous
    fields equal the current ones, as the reference's loader leaves them.
    """
    from .evolver import Evolver

    c = read_checkpoint(path)
    ev = Evolver(c["config"], backend=backend, buffers=buffers)
    ev.set_psi_real(c["psi_real"])
    if "psi_imag" in c:
        ev.set_psi_imag(c["psi_imag"])
    ev.set_chi(c["chi"])
    if c["exact"]:
        ev.set_psi_real_prev(c["leapfrog_psi_real_prev"])
        if "leapfrog_psi_imag_prev" in c:
            ev.set_psi_imag_prev(c["leapfrog_psi_imag_prev"])
        ev.set_chi_prev(c["leapfrog_chi_prev"])
    if "sa_fields" in c and getattr(ev, "_sa_on", False):
        ev.set_sa_fields(c["sa_fields"])
    ev.step = c["step"]
    return ev, c
