"""Host logic of the batched-replica workloads, without a GPU: the replica generator's
ranges and determinism, the 5-smooth mesh sizes, and each replica's parameters (the
one-image rule of the real-space sum: a box below twice the cutoff gets rc = L/2 and the
Ewald parameter raised to keep the truncation error at the tolerance).  The mesh sizes
decide the size groups whose transforms a lockstep batch runs as one batched plan."""
import math

import numpy as np


def test_replica_specs_ranges_and_determinism():
    from conductorrigid_b200 import systems

    specs = systems.replica_specs(256, seed=1)
    assert len(specs) == 256
    nb = np.array([s["n_bodies"] for s in specs])
    phi = np.array([s["phi"] for s in specs])
    field = np.array([s["field"] for s in specs])
    assert nb.min() >= 20 and nb.max() <= 400
    assert phi.min() >= 0.05 and phi.max() <= 0.35
    np.testing.assert_allclose(np.linalg.norm(field, axis=1), 1.0, atol=1e-12)
    assert len({s["seed"] for s in specs}) == 256
    again = systems.replica_specs(256, seed=1)
    assert again == specs
    assert systems.replica_specs(256, seed=2) != specs


def test_smooth_sizes():
    from conductorrigid_b200 import systems

    def smooth(m):
        for p in (2, 3, 5):
            while m % p == 0:
                m //= p
        return m == 1

    for n in range(1, 129):
        s = systems.smooth_at_least(n)
        assert smooth(s) and s >= n
        assert not any(smooth(k) for k in range(n, s))  # the smallest such size
    assert systems.smooth_at_least(129) == 128 and systems.smooth_at_least(1000) == 128  # the cap


def test_replica_params_and_size_groups(product_lib):
    from conductorrigid_b200 import batch, systems

    tol = 1e-5
    sizes = set()
    for sp in systems.replica_specs(256, seed=1):
        # the box edge of the replica, as systems.spheres derives it (unit spheres)
        L = (sp["n_bodies"] * 4.0 / 3.0 * math.pi / sp["phi"]) ** (1.0 / 3.0)
        grid = systems.smooth_at_least(int(math.ceil(2.0 * L)))
        sizes.add(grid)
        assert grid <= 128
    # the 256 replicas fall into a few size groups (cubic boxes: one size per replica)
    assert 5 <= len(sizes) <= 40
    for nb, phi in ((20, 0.33), (400, 0.05)):
        s = systems.spheres(np.ones(nb), 1, phi, (0.0, 0.0, 1.0), seed=3)
        p = batch.replica_params(s, tol=tol)
        L = float(min(s.L))
        rc = min(4.0, 0.5 * L * (1.0 - 1e-12))
        assert p.rcut == rc and p.xi == math.sqrt(-math.log(tol)) / rc
        assert tuple(p.grid) == tuple(systems.smooth_at_least(int(math.ceil(2.0 * Ld))) for Ld in s.L)
        assert p.support == 9 and p.precision == product_lib.CR_MIXED
    # a small box takes rc = L/2 below the default cutoff of 4
    s = systems.spheres(np.ones(20), 1, 0.33, (0.0, 0.0, 1.0), seed=3)
    assert batch.replica_params(s).rcut < 4.0
