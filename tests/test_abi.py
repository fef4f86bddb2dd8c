"""The C ABI without a GPU: the library loads, exports every declared symbol, and its
host-only parts (parameter derivation, tables, synthetic systems) agree with the
oracle bit for bit or to rounding."""
import ctypes as C
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent


def declared_symbols():
    names = []
    for hdr in sorted((ROOT / "include").glob("*.h")):
        text = hdr.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\*?\s*(cr_[a-z_0-9]+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_exports_every_declared_symbol(product_lib):
    names = declared_symbols()
    assert len(names) >= 25
    out = subprocess.run(["nm", "-D", "--defined-only", str(product_lib.LIB_PATH)], capture_output=True,
                         text=True).stdout
    exported = set(re.findall(r"\b(cr_[a-z_0-9]+)\b", out))
    missing = [n for n in names if n not in exported]
    assert not missing, missing
    L = C.CDLL(str(product_lib.LIB_PATH))
    for n in names:
        assert getattr(L, n) is not None
    # the Python binding covers the whole header
    assert set(names) <= set(product_lib.exported_symbols())


def test_abi_version_and_status(product_lib):
    lib = product_lib.lib()
    assert lib.cr_abi_version() == 5
    assert lib.cr_status_string(product_lib.CR_GRID_TOO_LARGE).decode() == "grid too large"


@pytest.mark.parametrize("case", range(4))
def test_derive_matches_oracle(product_lib, oracle_lib, case):
    from conductorrigid_b200.systems import XI_DEFAULT

    cases = [((16.12, 16.12, 16.12), 0.5, 1e-3, None, 0, 0.0), ((16.1199, 16.1199, 16.1199), XI_DEFAULT, 1e-5, 64, 9, 4.0),
             ((24.08, 24.08, 24.08), XI_DEFAULT, 1e-5, 128, 11, 4.0), ((30.0, 20.0, 12.0), 0.7, 1e-5, None, 0, 0.0)]
    L, xi, tol, grid, P, rc = cases[case]
    p = product_lib.make_params(xi=xi, errortol=tol, grid=grid, support=P, rcut=rc)
    d = product_lib.derive_params(p, L)
    o = oracle_lib.derive(L, xi, tol, grid, P, rc)
    assert list(d.grid) == list(o.N)
    assert d.support == o.P and d.support_unclamped == o.P_unclamped and d.n_table == o.N_table
    for a, b in [(d.h, o.h), (d.eta, o.eta)]:
        assert list(a) == list(b)
    assert (d.rcut, d.kcut, d.dr, d.xiterm, d.quadW) == (o.rc, o.kcut, o.dr, o.xiterm, o.quadW)
    assert d.prefac == pytest.approx(o.prefac, rel=1e-15)
    assert d.selfcoeff == pytest.approx(o.selfcoeff, rel=1e-15)
    t1, t2 = product_lib.build_tables(d, xi)
    o1, o2 = oracle_lib.tables(o)
    np.testing.assert_allclose(t1, o1, rtol=1e-14, atol=1e-16)
    np.testing.assert_allclose(t2, o2, rtol=1e-14, atol=1e-16)


def test_derive_errors(product_lib):
    lib = product_lib
    d = lib.CrDerived()
    L = np.array([10.0, 10.0, 10.0])
    for bad in [dict(xi=0.0), dict(errortol=0.0), dict(errortol=1.5), dict(rcut=6.0)]:
        p = lib.make_params(**{**dict(xi=0.9, errortol=1e-5), **bad})
        assert lib.lib().cr_derive_params(C.byref(p), lib.dptr(L), C.byref(d)) == lib.CR_BAD_PARAM
    # more than 4096 nodes per dimension (ConductorRigid.cc:181-189)
    p = lib.make_params(xi=40.0, errortol=1e-5)
    big = np.array([1000.0, 1000.0, 1000.0])
    assert lib.lib().cr_derive_params(C.byref(p), lib.dptr(big), C.byref(d)) == lib.CR_GRID_TOO_LARGE


def test_icosphere_and_placement(product_lib):
    from conductorrigid_b200 import systems

    assert [product_lib.lib().cr_util_icosphere_count(k) for k in range(3)] == [12, 42, 162]
    for lvl in (1, 2):
        v = systems.icosphere(lvl)
        np.testing.assert_allclose(np.linalg.norm(v, axis=1), 1.0, atol=1e-15)
        assert len(np.unique(np.round(v, 12), axis=0)) == len(v)
    w = systems.workload("polydisperse_204k", scale=0.02)
    s = w.system
    c, r = s.body_pos, s.radius
    d = c[:, None, :] - c[None, :, :]
    d -= s.L * np.rint(d / s.L)
    dist = np.linalg.norm(d, axis=-1)
    np.fill_diagonal(dist, np.inf)
    assert np.all(dist >= (r[:, None] + r[None, :]) - 1e-12)
    assert np.all(np.abs(s.pos) <= 0.5 * s.L[0])
    assert s.body_charge.sum() == 0 and set(np.unique(s.body_charge)) == {-1.0, 1.0}
    # the same seed gives the same system
    s2 = systems.workload("polydisperse_204k", scale=0.02).system
    assert np.array_equal(s.pos, s2.pos)


def test_compute_requires_topology(product_lib):
    """Host-side argument checks that run before any device work."""
    lib = product_lib.lib()
    d = C.c_void_p()
    assert lib.cr_destroy(None) == product_lib.CR_BAD_PARAM
    assert lib.cr_create(None, None, C.byref(d)) == product_lib.CR_BAD_PARAM


def test_lockstep_batch_argument_checks(product_lib):
    """The lockstep batch's host-side refusals (no device work): no handles, a null
    handle, a null batch; the creation message is readable with a NULL batch."""
    lib = product_lib.lib()
    out = C.c_void_p(1)
    assert lib.cr_batch_create(0, None, C.byref(out)) == product_lib.CR_BAD_PARAM
    assert not out.value
    assert b"no handles" in lib.cr_batch_last_error(None)
    assert lib.cr_batch_create(1, None, C.byref(out)) == product_lib.CR_BAD_PARAM
    assert lib.cr_batch_create(1, (C.c_void_p * 1)(None), None) == product_lib.CR_BAD_PARAM
    assert lib.cr_batch_create(1, (C.c_void_p * 1)(None), C.byref(out)) == product_lib.CR_BAD_PARAM
    assert not out.value and b"null handle" in lib.cr_batch_last_error(None)
    assert lib.cr_batch_destroy(None) == product_lib.CR_BAD_PARAM
    st = (product_lib.CrSolveStats * 1)()
    status = (C.c_int * 1)()
    assert lib.cr_batch_solve(None, None, None, None, None, None, st, status, 1) == product_lib.CR_BAD_PARAM
    a = C.c_longlong()
    assert lib.cr_batch_counters(None, C.byref(a), None, None) == product_lib.CR_BAD_PARAM
    x = C.c_double()
    assert lib.cr_batch_phase_ms(None, C.byref(x), None, None) == product_lib.CR_BAD_PARAM
