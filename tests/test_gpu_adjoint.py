"""Path-simulated portfolio loss and its adjoint (nmlmc_path_adjoint) on the GPU.

L_m against the CPU oracle (oracle/adjoint_oracle.c) on the same counter streams; FP32 paths
against FP64; the adjoint gradients of E[L] and of the sigmoid-smoothed P(L > K) against
central differences with common random numbers (the same seed on both sides, step 1e-4),
directly and through a torch.autograd.Function wrapper checked by torch.autograd.gradcheck.
"""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def small_portfolio(Q, P, seed, mu_eq_r=False):
    g = np.random.default_rng(seed)
    S0 = 100 * (1 + 0.1 * (g.random(Q) - 0.5))
    pf = dict(S0=S0, mu=np.full(Q, 0.05) if mu_eq_r else 0.02 + 0.08 * g.random(Q),
              sigma=0.1 + 0.3 * g.random(Q), stock_ind=g.integers(0, Q, P).astype(np.uint32),
              type=np.where(g.random(P) < 0.5, 1, -1).astype(np.int32),
              maturity=0.25 + 1.0 * g.random(P), w=g.standard_normal(P))
    pf["strike"] = S0[pf["stock_ind"]] * (0.85 + 0.3 * g.random(P))
    return pf


def batch_of(nm, sizes, seed=1, K=None, rho=0.2):
    pfs = [small_portfolio(Q, P, seed + k) for k, (Q, P) in enumerate(sizes)]
    return nm.make_batch(pfs, K if K is not None else [0.5] * len(sizes), r=0.05, rho=rho, tau=1 / 52)


@pytest.fixture(scope="module")
def sampler(nm):
    return nm.Sampler(precision=nm.PREC_FP64)


def test_loss_matches_oracle(nm, sampler):
    b = batch_of(nm, [(3, 40), (1, 7), (5, 25)])
    for ell, milstein in ((0, True), (3, True), (2, False)):
        g = sampler.path_adjoint(b, ell=ell, pairs=3, M=48, seed=11, milstein=milstein, grads=False,
                                 loss=True)
        o = O.adj_loss(b, ell, 3, 48, 11, milstein)
        scale = np.abs(o).max()
        np.testing.assert_allclose(g["loss"], o, rtol=1e-11, atol=1e-11 * scale)
        assert np.allclose(g["EL"], o.mean(axis=1), rtol=1e-12, atol=1e-12 * scale)
        np.testing.assert_allclose(g["P_hard"], (o > 0.5).mean(axis=1), rtol=1e-14)


def test_fp32_loss_bound(nm, sampler):
    """FP32 paths (SFU Box-Muller, float states) against FP64 on the same streams."""
    b = batch_of(nm, [(4, 300), (2, 50)])
    s32 = nm.Sampler(precision=nm.PREC_FP32)
    g64 = sampler.path_adjoint(b, ell=5, pairs=4, M=64, seed=3, grads=False, loss=True)
    g32 = s32.path_adjoint(b, ell=5, pairs=4, M=64, seed=3, grads=False, loss=True)
    oo = b["option_off"]
    for p in range(2):
        scale = np.abs(b["w"][oo[p]:oo[p + 1]]).sum() * 100.0   # sum |w_i| S0
        err = np.abs(g32["loss"][p] - g64["loss"][p]).max() / scale
        assert err < 5e-6, err


def test_batch_member_equals_single(nm, sampler):
    """Portfolio 0 of a batch draws the same streams as the same portfolio run alone."""
    pfs = [small_portfolio(3, 60, 5), small_portfolio(2, 30, 6)]
    b2 = nm.make_batch(pfs, [0.3, 0.3], rho=0.1)
    b1 = nm.make_batch(pfs[:1], [0.3], rho=0.1)
    g2 = sampler.path_adjoint(b2, ell=2, pairs=2, M=40, seed=9, loss=True)
    g1 = sampler.path_adjoint(b1, ell=2, pairs=2, M=40, seed=9, loss=True)
    np.testing.assert_allclose(g2["loss"][0], g1["loss"][0], rtol=1e-13, atol=1e-12)
    np.testing.assert_allclose(g2["grad_w_EL"][:60], g1["grad_w_EL"], rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(g2["grad_sigma_P"][:3], g1["grad_sigma_P"], rtol=1e-10, atol=1e-14)


def _perturbed(b, key, idx, h):
    c = dict(b)
    c[key] = np.array(b[key], dtype=np.float64).copy()
    c[key][idx] += h
    return c


def test_adjoint_matches_central_differences(nm, sampler):
    """dE[L]/dw_i, dP/dw_i, dE[L]/dsigma_j, dP/dsigma_j against CRN central differences."""
    b = batch_of(nm, [(3, 30), (2, 12)], seed=21, K=[0.0, 0.0])
    kw = dict(ell=3, pairs=2, M=128, seed=5, delta_rel=0.05)
    base = sampler.path_adjoint(b, loss=True, **kw)
    # threshold at the median loss so the smoothed probability has weight
    K = np.median(base["loss"], axis=1)
    b["K"] = K
    delta_abs = 0.05 * np.abs(K)
    g = sampler.path_adjoint(b, **kw)
    h = 1e-4

    def f(bb):
        r = sampler.path_adjoint(bb, grads=False, **kw)
        return r["EL"], r["P_smooth"]

    oo, so = b["option_off"], b["stock_off"]
    for i in [0, 3, 17, 29, 31, 41]:
        p = int(np.searchsorted(oo, i, side="right") - 1)
        ep, pp = f(_perturbed(b, "w", i, h))
        em, pm = f(_perturbed(b, "w", i, -h))
        np.testing.assert_allclose((ep[p] - em[p]) / (2 * h), g["grad_w_EL"][i], rtol=1e-8, atol=1e-10)
        np.testing.assert_allclose((pp[p] - pm[p]) / (2 * h), g["grad_w_P"][i], rtol=1e-4,
                                   atol=1e-6 / delta_abs[p])
    for j in range(int(so[-1])):
        p = int(np.searchsorted(so, j, side="right") - 1)
        ep, pp = f(_perturbed(b, "sigma", j, h))
        em, pm = f(_perturbed(b, "sigma", j, -h))
        fd_e, fd_p = (ep[p] - em[p]) / (2 * h), (pp[p] - pm[p]) / (2 * h)
        scale_e = np.abs(b["w"][oo[p]:oo[p + 1]]).sum() * 100.0
        assert abs(fd_e - g["grad_sigma_EL"][j]) <= 2e-3 * abs(g["grad_sigma_EL"][j]) + 1e-5 * scale_e, \
            (j, fd_e, g["grad_sigma_EL"][j])
        assert abs(fd_p - g["grad_sigma_P"][j]) <= 5e-3 * abs(g["grad_sigma_P"][j]) + 1e-4, \
            (j, fd_p, g["grad_sigma_P"][j])


def test_fp32_adjoint_close_to_fp64(nm, sampler):
    b = batch_of(nm, [(4, 200)], seed=31, K=[0.0])
    kw = dict(ell=4, pairs=4, M=256, seed=2)
    base = sampler.path_adjoint(b, loss=True, grads=False, **kw)
    b["K"] = np.median(base["loss"], axis=1)
    g64 = sampler.path_adjoint(b, **kw)
    g32 = nm.Sampler(precision=nm.PREC_FP32).path_adjoint(b, **kw)
    for k in ("grad_w_EL", "grad_sigma_EL"):
        np.testing.assert_allclose(g32[k], g64[k], rtol=2e-3, atol=1e-4 * np.abs(g64[k]).max())
    assert abs(g32["EL"][0] - g64["EL"][0]) < 1e-4 * np.abs(b["w"]).sum() * 100


def test_torch_autograd_gradcheck(nm, sampler):
    """torch.autograd.Function around the C-ABI: forward (E[L], P_delta), backward the adjoint;
    gradcheck's central differences run on common random numbers (fixed seed)."""
    torch = pytest.importorskip("torch")
    b0 = batch_of(nm, [(2, 8)], seed=41, K=[0.0])
    kw = dict(ell=2, pairs=2, M=64, seed=8, delta_rel=0.1)
    b0["K"] = np.median(sampler.path_adjoint(b0, loss=True, grads=False, **kw)["loss"], axis=1)

    class PathLoss(torch.autograd.Function):
        @staticmethod
        def forward(ctx, w, sigma):
            b = dict(b0, w=w.detach().numpy(), sigma=sigma.detach().numpy())
            r = sampler.path_adjoint(b, **kw)
            ctx.save_for_backward(torch.from_numpy(r["grad_w_EL"]), torch.from_numpy(r["grad_w_P"]),
                                  torch.from_numpy(r["grad_sigma_EL"]), torch.from_numpy(r["grad_sigma_P"]))
            return torch.tensor([r["EL"][0], r["P_smooth"][0]], dtype=torch.float64)

        @staticmethod
        def backward(ctx, go):
            gwE, gwP, gsE, gsP = ctx.saved_tensors
            return go[0] * gwE + go[1] * gwP, go[0] * gsE + go[1] * gsP

    w = torch.tensor(b0["w"], dtype=torch.float64, requires_grad=True)
    sg = torch.tensor(b0["sigma"], dtype=torch.float64, requires_grad=True)
    assert torch.autograd.gradcheck(PathLoss.apply, (w, sg), eps=1e-4, atol=2e-4, rtol=2e-3)


def test_invalid_arguments(nm, sampler):
    b = batch_of(nm, [(2, 5)])
    with pytest.raises(nm.NmlmcError):
        sampler.path_adjoint(b, ell=17, pairs=1, M=4)
    with pytest.raises(nm.NmlmcError):
        sampler.path_adjoint(b, ell=2, pairs=0, M=4)
    bad = dict(b, maturity=np.full(5, 0.001))
    with pytest.raises(nm.NmlmcError):
        sampler.path_adjoint(bad, ell=2, pairs=1, M=4)
