"""The finite-volume problem generators used by the differentiation tests:
the Jacobian J = d(values)/d(kappa) they return against central differences
of the values, and the values-only path against the full build."""

import numpy as np
import pytest

from draugr import problems

GENERATORS = {
    "fv_diffusion_3d": (lambda k, **kw: problems.fv_diffusion_3d(k, **kw), (5, 4, 6)),
    "convection_diffusion_2d": (lambda k, **kw: problems.convection_diffusion_2d(k, 50.0, seed=3, **kw),
                                (9, 9)),
}


@pytest.mark.parametrize("name", sorted(GENERATORS))
def test_jacobian_matches_central_differences(name):
    make, shape = GENERATORS[name]
    rng = np.random.default_rng(4)
    kappa = np.exp(rng.normal(0.0, 1.0, shape))
    A, J = make(kappa)
    assert J.shape == (A.nnz, kappa.size)
    eps = 1e-6
    for _ in range(5):
        delta = rng.normal(size=shape) * kappa
        vp = make(kappa + eps * delta, values_only=True)
        vm = make(kappa - eps * delta, values_only=True)
        fd = (vp - vm) / (2 * eps)
        ad = J @ delta.ravel()
        assert np.linalg.norm(fd - ad) <= 1e-7 * np.linalg.norm(ad)


@pytest.mark.parametrize("name", sorted(GENERATORS))
def test_values_only_equals_full_build(name):
    make, shape = GENERATORS[name]
    rng = np.random.default_rng(5)
    for _ in range(2):
        kappa = np.exp(rng.normal(0.0, 1.0, shape))
        A, _ = make(kappa)
        v = make(kappa, values_only=True)
        assert np.array_equal(v, A.data)


def test_convection_diffusion_is_a_nonsymmetric_m_matrix():
    kappa = np.exp(np.random.default_rng(6).normal(0.0, 1.0, (16, 16)))
    A, _ = problems.convection_diffusion_2d(kappa, 50.0, seed=1)
    d = A.diagonal()
    off = (A - np.diag(d)).toarray() if hasattr(A - np.diag(d), "toarray") else np.asarray(A - np.diag(d))
    assert abs(A - A.T).max() > 1.0
    assert (d > 0).all() and off.max() <= 0.0
    assert (d + off.sum(axis=1) >= -1e-12).all()  # weakly diagonally dominant rows
