"""The oracle-side system generator against the product's: identical arrays.

The CPU baseline and the reference-method arm of the benchmark build their inputs
through the oracle library alone (oracle/systems.py); the GPU arms through the
product's generator.  Both must describe the same systems bit for bit."""
import numpy as np
import pytest


@pytest.mark.parametrize("name,scale", [("plain_small", 1.0), ("precision_162k", 0.1), ("precision_162k", 1.0),
                                        ("polydisperse_204k", 0.05)])
def test_oracle_generator_matches_product(oracle_lib, product_lib, name, scale):
    from oracle import systems as osys

    from conductorrigid_b200 import systems

    a = systems.workload(name, seed=3, scale=scale)
    s, p = a.system, a.params
    o, op = osys.workload(name, seed=3, scale=scale)
    for k in ("L", "pos", "body", "rigid", "body_charge", "body_pos", "radius", "field"):
        x, y = getattr(s, k), getattr(o, k)
        assert x.dtype == y.dtype and x.shape == y.shape, k
        assert np.array_equal(x, y), k
    for k in ("xi", "errortol", "rcut", "grid", "support", "gmres_tol"):
        assert p[k] == op[k], k


def test_icosphere_and_uniform_match(oracle_lib, product_lib):
    from oracle import systems as osys

    from conductorrigid_b200 import systems

    for level in range(4):
        assert np.array_equal(systems.icosphere(level), osys.icosphere(level))
    assert np.array_equal(systems.uniform(12345, 1000), osys.uniform(12345, 1000))
    # a box smaller than three cells: the all-pairs branch
    r = np.array([1.0, 1.0, 0.5, 0.5, 0.5])
    assert np.array_equal(systems.place_spheres(r, [5.0, 5.0, 5.0], 9), osys.place_spheres(r, [5.0, 5.0, 5.0], 9))
