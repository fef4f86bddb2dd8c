"""Two-level preconditioner checker on the CPU: the dense restatement (coarse_ref) used as
the right preconditioner of FGMRES over the oracle's operator converges to the same
solution in far fewer iterations than the conductor response alone."""
import numpy as np


def _fgmres(matvec, prec, b, m=50, tol=1e-6, maxit=600):
    n = len(b)
    x = np.zeros(n)
    bn = np.linalg.norm(b)
    it = 0
    r = b.copy()
    while it < maxit:
        beta = np.linalg.norm(r)
        if beta <= tol * bn:
            break
        V = np.zeros((m + 1, n))
        Zs = np.zeros((m, n))
        H = np.zeros((m + 1, m))
        V[0] = r / beta
        g = np.zeros(m + 1)
        g[0] = beta
        cs, sn = np.zeros(m), np.zeros(m)
        j = 0
        for j in range(m):
            it += 1
            Zs[j] = prec(V[j])
            w = matvec(Zs[j])
            for _ in range(2):
                h = V[: j + 1] @ w
                w -= h @ V[: j + 1]
                H[: j + 1, j] += h
            H[j + 1, j] = np.linalg.norm(w)
            V[j + 1] = w / H[j + 1, j]
            for k in range(j):
                t = cs[k] * H[k, j] + sn[k] * H[k + 1, j]
                H[k + 1, j] = -sn[k] * H[k, j] + cs[k] * H[k + 1, j]
                H[k, j] = t
            den = np.hypot(H[j, j], H[j + 1, j])
            cs[j], sn[j] = H[j, j] / den, H[j + 1, j] / den
            H[j, j], H[j + 1, j] = den, 0.0
            g[j + 1] = -sn[j] * g[j]
            g[j] = cs[j] * g[j]
            if abs(g[j + 1]) <= tol * bn or it >= maxit:
                break
        k = j + 1
        y = np.linalg.solve(np.triu(H[:k, :k]), g[:k])
        x += y @ Zs[:k]
        r = b - matvec(x)
    return x, it


def test_two_level_reference_cuts_iterations(oracle_lib):
    from conductorrigid_b200 import systems
    from coarse_ref import TwoLevelRef

    s = systems.spheres(np.ones(40), 1, 0.30, (0.0, 0.0, 1.0), seed=5)
    o = oracle_lib.Oracle(s, systems.XI_DEFAULT, 1e-5, 32, 9, 4.0)
    pd = oracle_lib.params_dict(o.p)
    phiq, _ = oracle_lib.tables(o.p)
    ref = TwoLevelRef(s, dict(rcut=pd["rc"], dr=pd["dr"], n_table=pd["N_table"], selfcoeff=pd["selfcoeff"]),
                      phiq, systems.XI_DEFAULT)
    assert ref.C.shape == (3 * s.n_bodies, 3 * s.n_bodies)
    assert np.all(np.linalg.eigvalsh(0.5 * (ref.C + ref.C.T)) > 0)  # coarse operator SPD
    b = o.objective(s.field)
    x1, it1 = _fgmres(o.matvec, ref.conductor, b)
    x2, it2 = _fgmres(o.matvec, ref.apply, b)
    for x in (x1, x2):
        assert np.linalg.norm(b - o.matvec(x)) <= 1.01e-6 * np.linalg.norm(b)
    assert np.abs(x2 - x1).max() <= 1e-4 * np.abs(x1).max()
    print(f"\nconductor {it1} iterations, two-level {it2}")
    assert it2 * 2 <= it1


def test_sparse_coarse_solve_converges_to_dense(oracle_lib):
    """The CG steps of the sparse form approach the exact coarse inverse."""
    from conductorrigid_b200 import systems
    from coarse_ref import TwoLevelRef

    s = systems.spheres(np.ones(40), 1, 0.20, (0.0, 0.0, 1.0), seed=7)
    o = oracle_lib.Oracle(s, systems.XI_DEFAULT, 1e-5, 32, 9, 4.0)
    pd = oracle_lib.params_dict(o.p)
    phiq, _ = oracle_lib.tables(o.p)
    der = dict(rcut=pd["rc"], dr=pd["dr"], n_table=pd["N_table"], selfcoeff=pd["selfcoeff"])
    ref = TwoLevelRef(s, der, phiq, systems.XI_DEFAULT)
    g = np.random.default_rng(3).standard_normal(ref.C.shape[0])
    exact = ref.coarse_solve(g)
    errs = []
    for k in (2, 8, 40):
        ref.pcg_steps = k
        errs.append(np.linalg.norm(ref.coarse_solve(g) - exact) / np.linalg.norm(exact))
    print(f"\ncoarse CG steps 2 / 8 / 40: relative error {errs[0]:.1e} / {errs[1]:.1e} / {errs[2]:.1e}")
    assert errs[0] > errs[1] > errs[2] and errs[2] < 1e-4


def test_lower_tile_gauss_jordan_matches_inverse():
    """The coarse inverse's blocked Gauss-Jordan restated: 64-wide pivot blocks, only the
    128 x 128 tiles on and below the diagonal updated (upper tiles never read), panels
    completed by the sweep operator's sign rule, upper tiles mirrored at the end."""
    rng = np.random.default_rng(0)
    n, NB, GT = 384, 64, 128
    T = n // GT
    X = rng.standard_normal((n, n))
    C = X @ X.T + n * np.eye(n)
    A = C.copy()
    for tr in range(T):
        for tc in range(tr + 1, T):
            A[tr * GT:(tr + 1) * GT, tc * GT:(tc + 1) * GT] = np.nan  # must never be read

    def tile(i):
        return i // GT

    for k0 in range(0, n, NB):
        K = slice(k0, k0 + NB)
        tK = tile(k0)
        Dinv = np.linalg.inv(A[K, K])
        AK = np.stack([A[j, K] if tile(j) > tK else A[K, j] for j in range(n)], axis=1)
        R = Dinv @ AK
        R[:, K] = Dinv
        Fc = np.stack([-A[K, i] if tile(i) < tK else A[i, K] for i in range(n)], axis=0)
        An = A.copy()
        for tr in range(T):
            for tc in range(tr + 1):
                cols = np.arange(tc * GT, (tc + 1) * GT)
                for i in range(tr * GT, (tr + 1) * GT):
                    if k0 <= i < k0 + NB:
                        An[i, cols] = R[i - k0, cols]
                    else:
                        old = A[i, cols].copy()
                        old[(cols >= k0) & (cols < k0 + NB)] = 0.0
                        An[i, cols] = old - Fc[i] @ R[:, cols]
        A = An
    for tr in range(T):
        for tc in range(tr + 1, T):
            A[tr * GT:(tr + 1) * GT, tc * GT:(tc + 1) * GT] = A[tc * GT:(tc + 1) * GT, tr * GT:(tr + 1) * GT].T
    ref = np.linalg.inv(C)
    assert np.abs(A - ref).max() <= 1e-12 * np.abs(ref).max()
