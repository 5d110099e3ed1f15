"""CPU tests: the C-ABI library loads and exports every symbol include/tlbm.h
declares (no kernel launches), generated headers are current, lattice tables
agree with the oracle's, and the host-side validation raises TensorLBM's
exception types before any device work."""

from __future__ import annotations

import ctypes
import pathlib
import re
import subprocess

import numpy as np
import pytest
import torch

from oracle import lbm as O

ROOT = pathlib.Path(__file__).resolve().parents[1]


def _declared_symbols() -> list[str]:
    text = (ROOT / "include" / "tlbm.h").read_text()
    return re.findall(r"TLBM_API\s+[\w\s\*]+?\b(tlbm_\w+)\s*\(", text)


def test_header_declares_the_abi():
    names = _declared_symbols()
    assert "tlbm_step" in names and "tlbm_collide" in names and len(names) >= 20


def test_library_exports_every_declared_symbol():
    from tensorlbm_b200 import _lib

    lib = _lib.load()
    for name in _declared_symbols():
        assert hasattr(lib, name), name
    assert lib.tlbm_abi_version() == _lib.ABI_VERSION == 3
    assert lib.tlbm_status_string(3) == b"input and output buffers alias"
    # the Python binding types exactly the declared set
    assert sorted(_lib.exported_symbols()) == sorted(_declared_symbols())
    out = subprocess.run(["nm", "-D", "--defined-only", str(_lib.LIB_PATH)], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\b(tlbm_\w+)\b", out))
    assert set(_declared_symbols()) == exported


def test_struct_layouts_match_the_library():
    """The ctypes mirrors of tlbm_desc, tlbm_batch_domain and tlbm_batch_desc
    have the sizes the compiled library has."""
    import ctypes

    from tensorlbm_b200 import _lib

    lib = _lib.load()
    for which, cls in enumerate((_lib.Desc, _lib.BatchDomain, _lib.BatchDesc)):
        assert lib.tlbm_struct_size(which) == ctypes.sizeof(cls), cls.__name__
    assert lib.tlbm_struct_size(3) == -1


def test_argument_checks_without_gpu():
    """Status codes for bad arguments come back before any launch."""
    from tensorlbm_b200 import _lib, _ops

    lib = _lib.load()
    d = _ops.make_desc(19, (8, 8, 8), _lib.F32, _lib.COLL_BGK, 0.6)
    assert lib.tlbm_step(ctypes.byref(d), None, None, None, None, None, None, None) == _lib.ERR_ARG
    assert lib.tlbm_step(ctypes.byref(d), 16, 16, None, None, None, None, None) == _lib.ERR_ALIAS
    bad = _ops.make_desc(9, (8, 8, 2), _lib.F32, _lib.COLL_BGK, 0.6)
    assert lib.tlbm_step(ctypes.byref(bad), 16, 32, None, None, None, None, None) == _lib.ERR_SHAPE
    lid27 = _ops.make_desc(27, (8, 8, 8), _lib.F32, _lib.COLL_BGK, 0.6, bc=_lib.BC_LID)
    assert lib.tlbm_step(ctypes.byref(lid27), 16, 32, None, None, None, None, None) == _lib.ERR_UNSUPPORTED
    neg = _ops.make_desc(19, (8, 8, 8), _lib.F32, _lib.COLL_BGK, -1.0)
    assert lib.tlbm_step(ctypes.byref(neg), 16, 32, None, None, None, None, None) == _lib.ERR_ARG
    assert lib.tlbm_equilibrium(19, _lib.F16_SHIFTED, 10, 8, 8, 8, 8, 8, None) == _lib.ERR_DTYPE
    assert lib.tlbm_moving_lid(27, _lib.F32, 4, 4, 4, 8, 0.1, None) == _lib.ERR_UNSUPPORTED
    assert lib.tlbm_build_flags(10, None, None, 3, 8, None) == _lib.ERR_ARG
    assert lib.tlbm_link_blocks(0) == 0 and lib.tlbm_link_blocks(1025) == 2


def test_status_to_exception_mapping():
    from tensorlbm_b200 import _lib

    with pytest.raises(ValueError):
        _lib.check(_lib.ERR_SHAPE, "x")
    with pytest.raises(NotImplementedError):
        _lib.check(_lib.ERR_UNSUPPORTED, "x")
    with pytest.raises(RuntimeError):
        _lib.check(_lib.ERR_LAUNCH, "x")
    _lib.check(_lib.OK, "x")


def test_cpu_tensors_are_rejected():
    from tensorlbm_b200 import boundaries3d, d3q19, solver3d

    f = torch.rand((19, 4, 5, 6))
    with pytest.raises(RuntimeError, match="CUDA"):
        solver3d.collide_bgk3d(f, 0.6)
    with pytest.raises(RuntimeError, match="CUDA"):
        d3q19.macroscopic3d(f)
    with pytest.raises(RuntimeError, match="CUDA"):
        boundaries3d.sphere_mask(8, 8, 8, 4, 4, 4, 2, "cpu")


def test_generated_headers_are_current(tmp_path, monkeypatch):
    from tensorlbm_b200.csrc import gen_tables

    gen = ROOT / "tensorlbm_b200" / "csrc" / "generated"
    assert (gen / "lattice_tables.cuh").read_text() == gen_tables.gen_lattice_tables()
    assert (gen / "mrt_tables.cuh").read_text() == gen_tables.gen_mrt_header()


@pytest.mark.parametrize("q", [9, 19, 27])
def test_lattice_tables_match_oracle(q):
    from tensorlbm_b200 import lattice

    L = lattice.LATTICES[q]
    assert np.array_equal(L.c[:, : L.dim], O.C[q])
    assert np.array_equal(L.opp, O.opposite(q))
    assert np.allclose(L.w64, O.W64[q], rtol=0, atol=0)
    m, minv = lattice.mrt_matrices(q)
    assert np.array_equal(m, O.mrt_matrix(q))
    assert np.allclose(m @ minv, np.eye(q), atol=1e-12)


def test_d3q27_monomial_factorisation():
    """The 1-D factorised raw-moment transform of the kernels equals the 27x27 matrix."""
    M = O.monomial_matrix()
    c = O.C[27]
    rng = np.random.default_rng(0)
    f = rng.standard_normal(27)
    g = np.zeros((3, 3, 3))
    for q in range(27):
        g[c[q, 0] + 1, c[q, 1] + 1, c[q, 2] + 1] = f[q]
    for axis in range(3):
        g = np.moveaxis(g, axis, 0)
        vm, v0, vp = g[0].copy(), g[1].copy(), g[2].copy()
        g[0], g[1], g[2] = vm + v0 + vp, vp - vm, vp + vm
        g = np.moveaxis(g, 0, axis)
    m = np.array([g[a, b, d] for a, b, d in O.DEGREES])
    assert np.allclose(m, M @ f, atol=1e-12)


def test_periodic_bits():
    from tensorlbm_b200.boundary_registry import _periodic_bits

    assert _periodic_bits(False) == 0
    assert _periodic_bits(True) == 7
    assert _periodic_bits((True, False, False)) == 4  # (z, y, x)
    assert _periodic_bits({"y": True, "z": True, "x": False}) == 6
    with pytest.raises(ValueError):
        _periodic_bits((True, False))


def test_step_config_bits():
    from tensorlbm_b200 import _lib
    from tensorlbm_b200.solvers import StepConfig

    c = StepConfig(19, (4, 5, 6), 0.6, "mrt", u_in=0.04, rho_out=1.0)
    d = c.desc(_lib.F32)
    assert d.bc == _lib.BC_ZH_INLET | _lib.BC_ZH_OUTLET
    assert (d.nx, d.ny, d.nz) == (6, 5, 4)
    assert d.collision == _lib.COLL_MRT and abs(d.s_e - 1.19) < 1e-15 and d.s_pi == -1.0
    c2 = StepConfig(9, (5, 6), 0.6, "bgk", u_lid=0.1)
    d2 = c2.desc(_lib.F64)
    assert d2.bc == _lib.BC_LID and (d2.nx, d2.ny, d2.nz) == (6, 5, 1) and abs(d2.s_e - 1.64) < 1e-15


def test_sponge_strength_matches_reference():
    """make_sponge_strength (boundaries.py:388) on the CPU, bit for bit."""
    import numpy as np

    from tensorlbm_b200 import boundaries
    from tests.conftest import golden

    g = golden("far_field")
    s = boundaries.make_sponge_strength(8, 40, 25, 10, power=2.0)
    assert s.shape == (8, 40) and s.dtype == torch.float32
    assert np.array_equal(s.numpy(), g["sponge"])
