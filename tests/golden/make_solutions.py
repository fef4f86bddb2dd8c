"""Generate tests/golden/solution_<workload>.npz: oracle solutions at full size.

Each file holds the bead charges q and body potentials Phi of the named benchmark
workload (seed 1) solved by the FP64 oracle to a true relative residual of 1e-11
(oracle.Oracle.solve_tight: the oracle's own operator, ConductorRigid.cu:953-1020,
inside a block-preconditioned flexible GMRES), with the residual reached.  Systems
come from the oracle-side generator (oracle/systems.py), so nothing here loads the
CUDA product.  The GPU tests recompute the oracle residual of the stored solution
before they use it.

Run:  python tests/golden/make_solutions.py [workload ...]   (default: precision_162k)
"""
from __future__ import annotations

import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import oracle  # noqa: E402
from oracle import systems  # noqa: E402

OUT = Path(__file__).resolve().parent


def main(names):
    for name in names:
        s, p = systems.workload(name, seed=1)
        t0 = time.perf_counter()
        orc = oracle.Oracle(s, p["xi"], p["errortol"], p["grid"], p["support"], p["rcut"])
        ref = orc.solve_tight(s.field, tol=1e-11, restart=100, maxiter=4000)
        dt = time.perf_counter() - t0
        print(f"{name}: {s.n_beads} charges, {ref['iterations']} iterations, residual {ref['true_rel']:.3e}, "
              f"{dt:.0f} s on {oracle.lib().orc_num_threads()} threads", flush=True)
        np.savez_compressed(OUT / f"solution_{name}.npz", q=ref["q"], phi=ref["phi"],
                            residual=np.float64(ref["true_rel"]), iterations=np.int64(ref["iterations"]))


if __name__ == "__main__":
    main(sys.argv[1:] or ["precision_162k"])
