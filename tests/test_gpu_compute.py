"""The reference-surface force compute (Python -> pybind11 C++ class -> C ABI) on B200."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300))


@pytest.fixture(scope="module")
def small(cuda, product_lib, oracle_lib):
    from conductorrigid_b200 import systems

    w = systems.workload("plain_small", scale=0.3)
    s, p = w.system, w.params
    orc = oracle_lib.Oracle(s, p["xi"], p["errortol"], p["grid"], p["support"], p["rcut"])
    ref = orc.solve(s.field, restart=100, maxiter=4000, tol=1e-11)
    return s, p, ref


def test_compute_matches_oracle_and_writes_output(small, tmp_path):
    from conductorrigid_b200.compute import ConductorRigid

    s, p, ref = small
    prefix = str(tmp_path / "run")
    cr = ConductorRigid("all", s.body, s.body_charge, field=list(s.field), xi=p["xi"], errortol=p["errortol"],
                        fileprefix=prefix, period=5, system=s, grid=p["grid"], support=p["support"], rcut=p["rcut"],
                        gmres_tol=1e-7, restart=50, maxiter=4000, precision="mixed", precond="conductor")
    assert abs(cr.rcut - np.sqrt(-np.log(p["errortol"])) / p["xi"]) < 1e-12
    F = cr.compute(10)
    assert cr.stats["converged"] == 1
    assert rel(cr.charges, ref["q"]) < 1e-5
    assert rel(cr.potentials, ref["phi"]) < 1e-5
    assert rel(F, ref["force"]) < 1e-5
    # OutputData at timestep 10 (period 5, t0 0): three sections of N lines
    text = (tmp_path / "run.0000000010.txt").read_text().splitlines()
    N = s.n_beads
    assert text[0] == "Bead Position" and text[N + 1] == "Bead Charge" and text[2 * N + 2] == "Bead Force"
    assert len(text) == 3 * N + 3
    q = np.array([float(v) for v in text[N + 2:2 * N + 2]])
    assert rel(q, cr.charges) < 1e-9


def test_field_update_is_linear(small):
    from conductorrigid_b200.compute import ConductorRigid

    s, p, _ = small
    cr = ConductorRigid("all", s.body, s.body_charge, field=[0.0, 0.0, 1.0], xi=p["xi"], errortol=p["errortol"],
                        system=s, grid=p["grid"], support=p["support"], rcut=p["rcut"], gmres_tol=1e-9, restart=50,
                        maxiter=4000, precision="fp64", precond="conductor")
    cr.compute(0)
    q1 = cr.charges.copy()
    cr.update_field([0.0, 0.0, -2.0])
    cr.compute(1)
    assert rel(cr.charges, -2.0 * q1) < 1e-7
    cr.update_parameters([0.0, 0.0, 1.0], "", 0)
    cr.compute(2)
    assert rel(cr.charges, q1) < 1e-7
