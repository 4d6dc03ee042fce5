"""The FP64 direct-sum adjoint (the gradient oracle) against central finite differences of the
loss 1/2 sum |B(x_t) - B*_t|^2 with h = 1e-3 relative, for the current densities and the source
positions, with explicit and with the reference's azimuthal current directions. The loss is
quadratic in J, so plain central differences are exact there; in the positions the O(h^2) error is
removed by Richardson extrapolation of the h and h/2 differences."""
import numpy as np
import pytest

from oracle import oracle as O


def loss(src, w, J, tgt, Bstar, current):
    B = O.direct(src, w, J, tgt, current=current)
    return 0.5 * np.sum((B - Bstar) ** 2)


@pytest.mark.parametrize("azimuthal", [False, True])
def test_adjoint_matches_central_differences(azimuthal):
    rng = np.random.default_rng(5)
    n, m = 40, 25
    src = rng.normal(size=(n, 3))
    w = rng.uniform(0.5, 1.5, n)
    J = None if azimuthal else rng.normal(size=(n, 3))
    tgt = rng.normal(size=(m, 3)) * 2
    current = 1e6  # keep the loss well scaled
    Bstar = O.direct(src, w, J, tgt, current=current) * (1 + 0.05 * rng.normal(size=(m, 3)))
    g = O.direct(src, w, J, tgt, current=current) - Bstar
    dJ, dx = O.adjoint_direct(src, w, J, tgt, g, current=current)
    for q, d in [(0, 0), (7, 1), (19, 2), (33, 0)]:
        def central(h):
            sp, sm = src.copy(), src.copy()
            sp[q, d] += h
            sm[q, d] -= h
            return (loss(sp, w, J, tgt, Bstar, current) - loss(sm, w, J, tgt, Bstar, current)) / (2 * h)

        h = 1e-3 * max(abs(src[q, d]), 1e-3)
        fd = (4 * central(h / 2) - central(h)) / 3
        assert abs(fd - dx[q, d]) <= 1e-6 * max(abs(fd), 1e-12) + 1e-9 * np.abs(dx).max()
        if not azimuthal:
            h = 1e-3 * max(abs(J[q, d]), 1e-3)
            Jp, Jm = J.copy(), J.copy()
            Jp[q, d] += h
            Jm[q, d] -= h
            fd = (loss(src, w, Jp, tgt, Bstar, current) - loss(src, w, Jm, tgt, Bstar, current)) / (2 * h)
            assert abs(fd - dJ[q, d]) <= 1e-7 * max(abs(fd), 1e-12) + 1e-10 * np.abs(dJ).max()
