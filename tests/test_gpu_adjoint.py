"""Adjoint FMM (dLoss/dJ, dLoss/d(source positions)) through the C ABI against the FP64 direct-sum
adjoint of the oracle (itself checked against central differences on the CPU), and the
torch.autograd wrapper against finite differences."""
import numpy as np
import pytest

from bachelors_b200 import Plan, geometry as G
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def case(seed=3, azimuthal=False):
    xyz, w, J = G.torus(32, 16, 8, 2.0, 0.5, current="azimuthal" if azimuthal else "poloidal")
    rng = np.random.default_rng(seed)
    Jp = J * (1 + 0.05 * rng.normal(size=(len(J), 1)))
    tgt = G.uniform_points(1500, -3, 3, seed)
    return xyz, w, (None if azimuthal else Jp), tgt


# tolerances: the FMM truncation error at p = 12 (about 1e-6 for B here), loosened for FP32
@pytest.mark.parametrize("precision,tolJ,tolx", [("fp64", 5e-6, 2e-5), ("fp32", 2e-5, 1e-4)])
@pytest.mark.parametrize("azimuthal", [False, True])
def test_adjoint_matches_direct_adjoint(precision, tolJ, tolx, azimuthal):
    xyz, w, J, tgt = case(azimuthal=azimuthal)
    rng = np.random.default_rng(11)
    g = rng.normal(size=(len(tgt), 3))
    dt = np.float64 if precision == "fp64" else np.float32
    plan = Plan(order=12, leaf_capacity=32, precision=precision, m2l="simt")
    plan.set_sources(xyz.astype(dt), w.astype(dt), None if J is None else J.astype(dt))
    plan.set_targets(tgt.astype(dt))
    dJ, dx = plan.adjoint(g.astype(dt), current=2.0)
    x64 = xyz.astype(dt).astype(np.float64)
    rJ, rx = O.adjoint_direct(x64, w.astype(dt), None if J is None else J.astype(dt), tgt.astype(dt), g.astype(dt),
                              current=2.0)
    assert rel(dJ, rJ) < tolJ
    assert rel(dx, rx) < tolx
    # the 64 seeded coordinates of the differentiation benchmark, checked one by one
    idx = rng.choice(len(xyz), 64, replace=False)
    assert np.abs(dx[idx] - rx[idx]).max() < 10 * tolx * np.abs(rx).max()
    plan.close()


def test_adjoint_bf16x3_mode():
    xyz, w, J, tgt = case(seed=4)
    g = np.random.default_rng(2).normal(size=(len(tgt), 3))
    x, ww, JJ, t, gg = (a.astype(np.float32) for a in (xyz, w, J, tgt, g))
    plan = Plan(order=12, leaf_capacity=32, precision="fp32", m2l="bf16x3")
    plan.set_sources(x, ww, JJ)
    plan.set_targets(t)
    dJ, dx = plan.adjoint(gg)
    rJ, rx = O.adjoint_direct(x, ww, JJ, t, gg)
    assert rel(dJ, rJ) < 5e-5 and rel(dx, rx) < 2e-4


def test_autograd_wrapper_against_finite_differences():
    import torch
    from bachelors_b200.autograd import biot_savart
    xyz, w, J, tgt = case(seed=5)
    dev = "cuda"
    X = torch.tensor(xyz, dtype=torch.float64, device=dev, requires_grad=True)
    Wt = torch.tensor(w, dtype=torch.float64, device=dev)
    Jt = torch.tensor(J, dtype=torch.float64, device=dev, requires_grad=True)
    T = torch.tensor(tgt, dtype=torch.float64, device=dev)
    Bstar = torch.tensor(O.direct(xyz, w, J, tgt) * 1.01, device=dev)
    c, H = G.root_cube(xyz, tgt)
    from bachelors_b200 import Plan as P_
    plan = P_(order=16, leaf_capacity=32, precision="fp64", root=(c, H * 1.01))
    B = biot_savart(X, Wt, Jt, T, plan=plan)
    loss = 0.5 * ((B - Bstar) ** 2).sum()
    loss.backward()
    gx = X.grad.cpu().numpy()
    gJ = Jt.grad.cpu().numpy()
    # FP64 direct-sum adjoint of the same loss
    g = (B.detach() - Bstar).cpu().numpy()
    rJ, rx = O.adjoint_direct(xyz, w, J, tgt, g)
    assert rel(gJ, rJ) < 1e-7 and rel(gx, rx) < 1e-6

    def lossf(xx, jj):
        BB = O.direct(xx, w, jj, tgt)
        return 0.5 * np.sum((BB - Bstar.cpu().numpy()) ** 2)

    rng = np.random.default_rng(9)
    for q in rng.choice(len(xyz), 4, replace=False):
        d = int(rng.integers(3))
        h = 1e-3 * max(abs(xyz[q, d]), 1e-3)
        vals = []
        for hh in (h, h / 2):
            xp, xm = xyz.copy(), xyz.copy()
            xp[q, d] += hh
            xm[q, d] -= hh
            vals.append((lossf(xp, J) - lossf(xm, J)) / (2 * hh))
        fd = (4 * vals[1] - vals[0]) / 3
        assert abs(fd - gx[q, d]) <= 1e-5 * abs(fd) + 1e-9 * np.abs(gx).max()


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("fp32", 1e-5)])
@pytest.mark.parametrize("with_J", [True, False])
def test_adjoint_direct_matches_oracle(precision, tol, with_J):
    from bachelors_b200 import Plan, geometry as G
    from oracle import oracle as O
    xyz, w, J = G.torus(16, 8, 4, 2.0, 0.5)
    tgt = G.uniform_points(700, -3, 3, 4)
    g = np.random.default_rng(8).normal(size=tgt.shape)
    dt = np.float64 if precision == "fp64" else np.float32
    plan = Plan(order=4, leaf_capacity=32, precision=precision)
    plan.set_sources(xyz.astype(dt), w.astype(dt), J.astype(dt) if with_J else None)
    plan.set_targets(tgt.astype(dt))
    dJ, dx = plan.adjoint_direct(g.astype(dt), 1.7)
    rJ, rx = O.adjoint_direct(xyz, w, J if with_J else None, tgt, g, current=1.7)
    assert np.linalg.norm(dJ - rJ) / np.linalg.norm(rJ) < tol
    assert np.linalg.norm(dx - rx) / np.linalg.norm(rx) < tol
    plan.close()


def test_autograd_gradcheck_fp64():
    """torch.autograd.gradcheck of the wrapper in FP64 on a small problem: the adjoint FMM's
    Jacobian-vector products against finite differences of the forward FMM (positions and J)."""
    import torch
    from bachelors_b200 import Plan
    from bachelors_b200.autograd import biot_savart
    xyz, w, J = G.torus(8, 4, 2, 2.0, 0.5)
    rng = np.random.default_rng(11)
    tgt = rng.normal(size=(6, 3))
    tgt = tgt / np.linalg.norm(tgt, axis=1, keepdims=True) * 6.0
    c, H = G.root_cube(xyz, tgt)
    plan = Plan(order=16, leaf_capacity=8, precision="fp64", root=(c, H * 1.01))
    X = torch.tensor(xyz, dtype=torch.float64, device="cuda", requires_grad=True)
    Jt = torch.tensor(J, dtype=torch.float64, device="cuda", requires_grad=True)
    Wt = torch.tensor(w, dtype=torch.float64, device="cuda")
    T = torch.tensor(tgt, dtype=torch.float64, device="cuda")
    f = lambda x, j: biot_savart(x, Wt, j, T, plan=plan) * 1e7   # scale B (~1e-7 T) to O(1)
    assert torch.autograd.gradcheck(f, (X, Jt), eps=1e-6, atol=1e-5, rtol=1e-3)
    plan.close()


def test_autograd_backward_after_plan_reuse():
    """Two forwards on one plan, then backward of the first: the gradients are those of the first
    problem (the wrapper restores its inputs when the plan has been given others since)."""
    import torch
    from bachelors_b200 import Plan
    from bachelors_b200.autograd import biot_savart
    xyz, w, J = G.torus(16, 8, 4, 2.0, 0.5)
    rng = np.random.default_rng(5)
    t1 = rng.uniform(-3, 3, size=(200, 3))
    t2 = rng.uniform(-3, 3, size=(150, 3))
    d = lambda a, g=False: torch.tensor(a, dtype=torch.float64, device="cuda", requires_grad=g)
    plan = Plan(order=10, leaf_capacity=16, precision="fp64")
    X1, J1 = d(xyz, True), d(J, True)
    B1 = biot_savart(X1, d(w), J1, d(t1), plan=plan)
    X2, J2 = d(xyz * 1.1, True), d(J * 0.5, True)
    B2 = biot_savart(X2, d(w), J2, d(t2), plan=plan)
    g1 = d(rng.normal(size=t1.shape))
    (B1 * g1).sum().backward()
    ref = Plan(order=10, leaf_capacity=16, precision="fp64")
    ref.set_sources(xyz, w, J)
    ref.set_targets(t1)
    rJ, rX = ref.adjoint_direct(g1.cpu().numpy())
    ref.close()
    # the adjoint FMM's accuracy at p = 10; the second problem's gradients differ by O(1)
    assert np.linalg.norm(J1.grad.cpu().numpy() - rJ) / np.linalg.norm(rJ) < 5e-5
    assert np.linalg.norm(X1.grad.cpu().numpy() - rX) / np.linalg.norm(rX) < 5e-5
    assert B2.shape == (150, 3)
    plan.close()


def test_autograd_gradcheck_azimuthal_current_fp64():
    """J = None (the reference's azimuthal direction): no gradient for J, and the position gradient
    includes the direction's dependence on the source positions (gradcheck in FP64)."""
    import torch
    from bachelors_b200 import Plan
    from bachelors_b200.autograd import biot_savart
    xyz, w, _ = G.torus(8, 4, 2, 2.0, 0.5, current="azimuthal")
    rng = np.random.default_rng(12)
    tgt = rng.normal(size=(6, 3))
    tgt = tgt / np.linalg.norm(tgt, axis=1, keepdims=True) * 6.0
    c, H = G.root_cube(xyz, tgt)
    plan = Plan(order=16, leaf_capacity=8, precision="fp64", root=(c, H * 1.01))
    X = torch.tensor(xyz, dtype=torch.float64, device="cuda", requires_grad=True)
    Wt = torch.tensor(w, dtype=torch.float64, device="cuda")
    T = torch.tensor(tgt, dtype=torch.float64, device="cuda")
    f = lambda x: biot_savart(x, Wt, None, T, plan=plan) * 1e7
    assert torch.autograd.gradcheck(f, (X,), eps=1e-6, atol=1e-5, rtol=1e-3)
    plan.close()
