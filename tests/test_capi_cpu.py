"""C ABI checks that need no GPU: the library builds, loads, exports every
function include/lfm_b200.h declares, and its host-side mask table is exact."""

from __future__ import annotations

import re

import numpy as np
import pytest

from conftest import ROOT, load_golden


@pytest.fixture(scope="module")
def lib():
    from lfm_b200 import _lib
    from lfm_b200.build import build_library

    build_library()
    return _lib.load()


def header_functions() -> list[str]:
    text = (ROOT / "include" / "lfm_b200.h").read_text()
    return sorted(set(re.findall(r"^\s*(?:const\s+char\*|int)\s+(lfm_\w+)\s*\(", text, re.M)))


def test_header_declares_the_abi():
    names = header_functions()
    for must in ("lfm_step_real_f32", "lfm_step_complex_f32", "lfm_step_color_f32",
                 "lfm_leapfrog_real_f32", "lfm_helmholtz_sa_f32", "lfm_mask_lut_build"):
        assert must in names


def test_library_exports_every_declared_function(lib):
    from lfm_b200 import _lib

    missing = [n for n in header_functions() if not hasattr(lib, n)]
    assert not missing, f"not exported: {missing}"
    # the Python binding covers the whole header
    assert set(header_functions()) <= set(_lib.exported_symbols())
    assert lib.lfm_abi_version() == 1


def header_arity() -> dict:
    """Parameter count of every function the header declares."""
    text = (ROOT / "include" / "lfm_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    out = {}
    for m in re.finditer(r"^\s*(?:const\s+char\*|int)\s+(lfm_\w+)\s*\(([^;]*?)\)\s*;", text,
                         re.M | re.S):
        params = m.group(2).strip()
        out[m.group(1)] = 0 if params in ("", "void") else params.count(",") + 1
    return out


def test_binding_signatures_match_the_header(lib):
    from lfm_b200 import _lib

    arity = header_arity()
    assert len(arity) >= 20
    for name, args in _lib._SIGNATURES.items():
        assert name in arity, name
        assert len(args) == arity[name], (name, len(args), arity[name])


def test_strerror_names_codes(lib):
    assert lib.lfm_strerror(0) == b"ok"
    assert lib.lfm_strerror(6).startswith(b"mask")


@pytest.mark.parametrize("N", [8, 12, 13, 16, 33, 64, 96])
@pytest.mark.parametrize("bf", [0.15, 0.3, 0.5])
def test_mask_table_reproduces_mask_exactly(lib, N, bf):
    from lfm_b200.mask import MaskTable, boundary_mask, radial_keys

    m = boundary_mask(N, bf)
    t = MaskTable.from_mask(N, m)
    assert t.desc.shift == (3 if N % 2 == 0 else 2)
    got = t.lookup(radial_keys(N))
    assert np.array_equal(got.view(np.uint32), m.view(np.uint32))
    # the table is small: the sponge band only
    assert t.table.size <= (3 * N * N) // 4 + 16


def test_mask_matches_reference_fixture(lib):
    import hashlib
    import json

    from lfm_b200.mask import MaskTable, boundary_mask, radial_keys

    g = load_golden("masks.npz")
    for key, ref in g.items():
        if key.startswith("mask_"):
            _, N, bf = key.split("_")
            assert np.array_equal(boundary_mask(int(N), float(bf)), ref), key
    for key, h in json.loads(str(g["large_mask_sha256"])).items():
        N, bf = int(key.split("_")[0]), float(key.split("_")[1])
        assert hashlib.sha256(boundary_mask(N, bf).tobytes()).hexdigest() == h, key
        # the formula-built table gives the same bits through the key lookup
        t = MaskTable.for_lattice(N, bf)
        assert hashlib.sha256(t.lookup(radial_keys(N)).tobytes()).hexdigest() == h, key


@pytest.mark.parametrize("N", [8, 13, 16, 33, 64])
@pytest.mark.parametrize("bf", [0.15, 0.3, 0.5, 0.9])
def test_formula_table_equals_scanned_table(lib, N, bf):
    from lfm_b200.mask import MaskTable, boundary_mask, radial_keys

    a = MaskTable.for_lattice(N, bf)
    b = MaskTable.from_mask(N, boundary_mask(N, bf))
    q = radial_keys(N)
    assert np.array_equal(a.lookup(q).view(np.uint32), b.lookup(q).view(np.uint32))


def test_mask_table_rejects_non_radial_mask(lib):
    from lfm_b200._lib import LFM_ERR_MASK, LfmError
    from lfm_b200.mask import MaskTable, boundary_mask

    m = boundary_mask(16, 0.3).copy()
    band = np.flatnonzero((m > 0) & (m < 1))
    m[band[0]] = 0.123  # break radial symmetry
    with pytest.raises(LfmError) as e:
        MaskTable.from_mask(16, m)
    assert e.value.code == LFM_ERR_MASK


def test_mask_table_edge_cases(lib):
    from lfm_b200.mask import MaskTable, radial_keys

    N = 10
    zero = MaskTable.from_mask(N, np.zeros(N**3, np.float32))
    assert (zero.lookup(radial_keys(N)) == 0).all()
    assert zero.desc.count == 0 and zero.desc.q_hi < zero.desc.q_lo
    one = MaskTable.from_mask(N, np.ones(N**3, np.float32))
    assert (one.lookup(radial_keys(N)) == 1).all()


def _clamped_key_mask(N: int, desc, table: np.ndarray) -> np.ndarray:
    """The step kernels' shared-memory sponge lookup, in int32 as the kernel
    computes it (csrc/step_tma.cu: key_shift, sponge_key, tab_mask, min_relu):
    a table [0, table..., 1] indexed by a byte offset clamped to
    [0, 4 * (count + 1)], the offset a sum of per-axis terms qterm >> shift."""
    i32 = np.int32
    sh = 2 if N % 2 else 3
    x = np.arange(N, dtype=i32)
    term4 = (4 * ((2 * x - N + 1) ** 2 >> sh)).astype(i32)
    key_lo = i32(min(int(desc.q_lo), 3 * N * N) >> sh)
    aj4 = (term4 + 4 * (1 - key_lo)).astype(i32)
    cap4 = i32(4 * (desc.count + 1))
    with np.errstate(over="raise"):
        off = term4[:, None, None] + aj4[None, :, None] + term4[None, None, :]
    assert off.dtype == np.int32
    off = np.maximum(np.minimum(off, cap4), 0)
    tab = np.concatenate([[0.0], table[: desc.count], [1.0]]).astype(np.float32)
    return tab[off >> 2].ravel()


@pytest.mark.parametrize("N", [8, 9, 16, 21, 36, 64])
@pytest.mark.parametrize("bf", [0.1, 0.3, 0.7])
def test_clamped_key_lookup_reproduces_the_mask(lib, N, bf):
    from lfm_b200.mask import MaskTable, boundary_mask

    m = boundary_mask(N, bf)
    t = MaskTable.from_mask(N, m)
    assert np.array_equal(_clamped_key_mask(N, t.desc, t.table).view(np.uint32), m.view(np.uint32))
    f = MaskTable.for_lattice(N, bf)
    assert np.array_equal(_clamped_key_mask(N, f.desc, f.table).view(np.uint32), m.view(np.uint32))


def test_clamped_key_lookup_empty_bands_and_range(lib):
    from lfm_b200.mask import MaskTable

    for N in (12, 13):
        for fill in (0.0, 1.0):
            t = MaskTable.from_mask(N, np.full(N**3, fill, np.float32))
            assert (_clamped_key_mask(N, t.desc, t.table) == fill).all()
    # offsets stay inside int32 up to the largest lattice (q_lo capped at 3 N^2)
    i32 = np.iinfo(np.int32)
    for N in (511, 512, 2047, 2048):
        sh = 2 if N % 2 else 3
        key_max = (3 * (N - 1) ** 2) >> sh
        for q_lo in (i32.max, 3, 0):
            key_lo = min(q_lo, 3 * N * N) >> sh
            lo, hi = 4 * (1 - key_lo), 4 * (key_max + 1 - key_lo)
            assert i32.min <= lo and hi <= i32.max


def test_bad_sizes_are_rejected(lib):
    import ctypes

    from lfm_b200._lib import LFM_ERR_CAPACITY, LFM_ERR_INVALID_ARG, LfmError, MaskLut, call
    from lfm_b200.mask import boundary_mask

    d = MaskLut()
    with pytest.raises(LfmError) as e:
        call("lfm_mask_lut_build", 1, None, None, 0, ctypes.byref(d))
    assert e.value.code == LFM_ERR_INVALID_ARG
    m = boundary_mask(16, 0.3)
    tiny = np.zeros(2, np.float32)
    with pytest.raises(LfmError) as e:
        call("lfm_mask_lut_build", 16, m.ctypes.data, tiny.ctypes.data, 2, ctypes.byref(d))
    assert e.value.code == LFM_ERR_CAPACITY
    with pytest.raises(LfmError) as e:
        call("lfm_step_real_f32", *([None] * 9), 16, 4e-4, 1 / 63, 0.0, 19.0, 0.0, None)
    assert e.value.code == LFM_ERR_INVALID_ARG


def test_config_validation_matches_reference_rules():
    from lfm_b200.config import FieldLevel, SimulationConfig, full_physics, gravity_only

    with pytest.raises(ValueError, match="grid_size"):
        SimulationConfig(grid_size=4)
    with pytest.raises(ValueError, match="CFL"):
        SimulationConfig(dt=0.06)
    with pytest.raises(ValueError, match="boundary_fraction"):
        SimulationConfig(boundary_fraction=1.0)
    c = gravity_only(64)
    assert c.field_level == FieldLevel.REAL and c.kappa == pytest.approx(1 / 63)
    f = full_physics(32)
    assert f.sa_enabled and f.lambda_self == pytest.approx(4 / 31)
    assert f.kappa_tube == pytest.approx(30 / 63) and f.sa_d == pytest.approx(4.9)


def test_product_does_not_import_the_oracle():
    pkg = ROOT / "lfm-physics_b200"
    for p in list(pkg.rglob("*.py")) + list(pkg.rglob("*.cu")) + list(pkg.rglob("*.cuh")):
        text = p.read_text()
        assert not re.search(r"(from|import)\s+oracle|lfm_oracle|oracle/", text), p


def test_every_python_source_compiles():
    """Every module of the package, the tests, the oracle and bench.py byte-compile (a
    syntax error in a GPU-only module would otherwise surface only on the GPU machine)."""
    import py_compile
    import tempfile
    from pathlib import Path

    root = Path(__file__).resolve().parents[1]
    files = [root / "bench.py", root / "__graft_entry__.py"]
    for d in ("lfm-physics_b200/lfm_b200", "tests", "tests/golden", "oracle"):
        files += sorted((root / d).glob("*.py"))
    with tempfile.TemporaryDirectory() as tmp:
        for i, f in enumerate(files):
            py_compile.compile(str(f), cfile=str(Path(tmp) / f"{i}.pyc"), doraise=True)
