"""cr_virial against the NumPy restatement of the virial (tests/virial_ref.py, itself
checked against finite differences of the oracle's energy in tests/test_virial.py)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("scale,support", [(0.3, 9), (1.0, 11)])
def test_virial_matches_restatement(cuda, product_lib, oracle_lib, scale, support):
    from conductorrigid_b200 import systems
    from conductorrigid_b200.device import Handle
    from tests import virial_ref as vr

    w = systems.workload("plain_small", seed=2, scale=scale)
    s, p = w.system, w.params
    orc = oracle_lib.Oracle(s, p["xi"], p["errortol"], p["grid"], support, p["rcut"])
    h = Handle(product_lib.make_params(field=tuple(s.field), xi=p["xi"], errortol=p["errortol"], grid=p["grid"],
                                       support=support, rcut=p["rcut"]), s.L)
    h.set_topology(s.body, s.rigid, s.body_charge)
    h.set_positions(s.pos, s.body_pos)
    q = np.random.default_rng(7).standard_normal(s.n_beads)
    v = h.virial(q)
    Vr = vr.real_virial(orc.p, s.pos, s.L, q)
    Vw, Ew = vr.wave_virial(orc.p, s.pos, s.L, q)
    assert np.abs(v["real"] - Vr).max() <= 1e-11 * np.abs(Vr).max()
    assert np.abs(v["wave"] - Vw).max() <= 1e-10 * np.abs(Vw).max()
    assert abs(v["wave_energy"] - Ew) <= 1e-11 * abs(Ew)
    assert abs(v["wave_energy"] - 0.5 * float(q @ h.wave_potential(q).cpu().numpy())) <= 1e-11 * abs(Ew)
    h.close()
