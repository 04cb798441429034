"""The host CMA-ES (tetris_ai3_b200/host/cmaes.cpp) against the reference's
own optimiser tests: ta3_trainer/tests/src/pagmo/dd_cmaes_test.cpp:22-104 and
sep_cmaes_test.cpp:22-80 (dim 10, box [-5, 5], population 12, sigma0 0.5,
ftol = xtol = 1e-14, champion below 1e-6), plus the eigensolver, the ask/tell
contract and the state round trip."""
from __future__ import annotations

import numpy as np
import pytest

DD_SEED, SEP_SEED = 0xDD5, 0x5E9


@pytest.mark.parametrize("problem,gens", [(0, 400), (1, 700), (2, 1500)])
def test_dd_converges_like_the_reference(host, problem, gens):
    f, x = host.run_test_problem(host.DD, problem, gens, seed=DD_SEED)
    assert f < 1e-6, (problem, f)


@pytest.mark.parametrize("problem,gens", [(0, 400), (1, 600)])
def test_sep_converges_like_the_reference(host, problem, gens):
    f, x = host.run_test_problem(host.SEP, problem, gens, seed=SEP_SEED)
    assert f < 1e-6, (problem, f)


def test_sep_cannot_learn_rotations_but_dd_can(host):
    # sep_cmaes_test.cpp:34-37: rotated problems are out of scope for the diagonal model
    f_sep, _ = host.run_test_problem(host.SEP, 2, 1500, seed=SEP_SEED)
    f_dd, _ = host.run_test_problem(host.DD, 2, 1500, seed=DD_SEED)
    assert f_dd < 1e-6 < f_sep


@pytest.mark.parametrize("kind", [1, 2])
def test_deterministic_for_seed(host, kind):
    a = host.run_test_problem(kind, 0, 30, seed=7)
    b = host.run_test_problem(kind, 0, 30, seed=7)
    c = host.run_test_problem(kind, 0, 30, seed=8)
    assert a[0] == b[0] and np.array_equal(a[1], b[1])
    assert not np.array_equal(a[1], c[1])


def test_jacobi_eigensolver_matches_numpy(host):
    rng = np.random.default_rng(3)
    for n in (1, 2, 10, 97):
        m = rng.normal(size=(n, n))
        a = m + m.T
        w, v, ok = host.sym_eig(a)
        assert ok
        ref = np.linalg.eigvalsh(a)
        assert np.allclose(np.sort(w), ref, rtol=1e-10, atol=1e-10 * np.abs(ref).max())
        assert np.allclose(v @ np.diag(w) @ v.T, a, atol=1e-9 * np.abs(a).max())
        assert np.allclose(v.T @ v, np.eye(n), atol=1e-10)


@pytest.mark.parametrize("kind", [1, 2])
def test_ask_tell_contract(host, kind):
    n = 6
    cma = host.Cma(kind, np.zeros(n), -np.ones(n), np.ones(n), 0.3, 11)
    x = cma.ask(8)
    assert x.shape == (8, n) and np.isfinite(x).all()
    # the initial per-axis std is sigma0 * box width
    assert np.allclose(cma.axis_std(), 0.3 * 2.0)
    with pytest.raises(ValueError):
        cma.tell(np.zeros(9))              # more values than asked
    with pytest.raises(ValueError):
        cma.tell(np.zeros(5), idx=[0, 1, 2, 3, 8])
    with pytest.raises(ValueError):
        cma.ask(4)                         # the reference needs >= 5 individuals
    f = (x ** 2).sum(1)
    cma.tell(f)
    best = x[np.argmin(f)]
    # the mean moves toward the better half
    assert np.linalg.norm(cma.mean - best) < np.linalg.norm(best) + 1e-12 or np.linalg.norm(cma.mean) < 1.0


@pytest.mark.parametrize("kind", [1, 2])
def test_subset_tell_uses_only_the_evaluated_candidates(host, kind):
    n = 5
    a = host.Cma(kind, np.zeros(n), -np.ones(n), np.ones(n), 0.5, 5)
    b = host.Cma(kind, np.zeros(n), -np.ones(n), np.ones(n), 0.5, 5)
    xa, xb = a.ask(12), b.ask(12)
    assert np.array_equal(xa, xb)
    idx = np.array([3, 0, 7, 11, 5, 9])
    f = (xa[idx] ** 2).sum(1)
    a.tell(f, idx=idx)
    # same candidates asked in that order then told as a full batch of a 6-candidate ask
    c = host.Cma(kind, np.zeros(n), -np.ones(n), np.ones(n), 0.5, 5)
    c.ask(12)
    c.tell(f, idx=idx)
    assert np.array_equal(a.mean, c.mean) and a.sigma == c.sigma
    assert not np.array_equal(a.mean, np.zeros(n))


@pytest.mark.parametrize("kind", [1, 2])
def test_saved_state_resumes_identically(host, kind):
    # dd_cmaes_test.cpp:82-104: a restored optimiser continues exactly like the original
    n = 10
    rot = np.linalg.qr(np.random.default_rng(0xDD).normal(size=(n, n)))[0]
    scale = 1e6 ** (np.arange(n) / (n - 1))
    fit = lambda X: ((X @ rot.T) ** 2 * scale).sum(1)
    cma = host.Cma(kind, np.full(n, 1.0), -5 * np.ones(n), 5 * np.ones(n), 0.5, 0xDD5)
    cma.new_evolve()
    for _ in range(40):
        x = cma.ask(12)
        cma.tell(fit(x))
    blob = cma.save()
    assert blob[:8] == b"TA3CMAES"
    twin = host.Cma.load(blob)
    for _ in range(25):
        x1, x2 = cma.ask(12), twin.ask(12)
        assert np.array_equal(x1, x2)
        cma.tell(fit(x1))
        twin.tell(fit(x2))
    assert np.array_equal(cma.mean, twin.mean) and cma.sigma == twin.sigma
    with pytest.raises(ValueError):
        host.Cma.load(b"not a state")
    with pytest.raises(ValueError):
        host.Cma.load(blob[:-9])


def test_nan_fitness_ranks_last(host):
    n = 4
    a = host.Cma(2, np.zeros(n), -np.ones(n), np.ones(n), 0.5, 1)
    b = host.Cma(2, np.zeros(n), -np.ones(n), np.ones(n), 0.5, 1)
    xa, xb = a.ask(10), b.ask(10)
    f = (xa ** 2).sum(1)
    worst = np.argsort(f)[-3:]
    g = f.copy()
    g[worst] = np.nan                     # NaN sorts after every number (dd_cmaes.cpp:26-32)
    f2 = f.copy()
    f2[worst] = f.max() + np.array([1.0, 2.0, 3.0])[np.argsort(np.argsort(f[worst]))]
    a.tell(g)
    b.tell(f2)
    assert np.allclose(a.mean, b.mean)


@pytest.mark.parametrize("kind", ["SEP", "DD"])
def test_whiten_maps_samples_to_a_standard_normal(host, kind):
    """Whitening inverts ask's sampling map: after some adaptation (an anisotropic, rotated
    distribution for dd-CMA-ES), a large sample is N(0, I) in the whitened coordinates."""
    import numpy as np
    dim = 10
    rng = np.random.default_rng(1)
    rot = np.linalg.qr(rng.normal(size=(dim, dim)))[0]
    scale = np.logspace(0, 2, dim)
    opt = host.Cma(getattr(host, kind), np.full(dim, 0.5), np.full(dim, -5.0), np.full(dim, 5.0), 0.5, 7)
    for _ in range(30):                                   # rotated ellipsoid: the distribution adapts
        x = opt.ask(12)
        f = (((x @ rot) * scale) ** 2).sum(1)
        opt.tell(f)
    x = opt.ask(20000)
    z = opt.whiten(x)
    assert np.abs(z.mean(0)).max() < 0.05
    assert np.abs(np.cov(z.T) - np.eye(dim)).max() < 0.08
