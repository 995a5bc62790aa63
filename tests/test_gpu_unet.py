"""GPU tests of the learned preconditioner (k_unet.cu): the U-Net forward pass
and the gradients of both training losses against a plain PyTorch restatement
(tests/unet_ref.py) of the same BF16-activation network, a directional
finite-difference check of the device gradient, training, and the A/B test of
the learned preconditioner inside FGMRES against the Jacobi one.
Tolerances: forward 1e-2 relative L2 (BF16 activations, FP32 accumulation in a
different order), gradients 5e-2 relative L2 per convolution."""
import numpy as np
import pytest

from hicar_b200 import _capi, cases

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

NX, NY, NZ = 70, 37, 6  # odd x-y sizes exercise the pooling edges and ragged conv tiles


@pytest.fixture(autouse=True)
def _fresh(lib):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from hicar_b200 import wind, wind_iterative
    wind_iterative.finalize_iter_winds()
    wind.reset()
    yield
    wind_iterative.finalize_iter_winds()
    wind.reset()


def _net_and_input(seed=0):
    from hicar_b200 import learned as L
    net = L.UNet(NX, NY, NZ, seed=seed)
    p = net.params().cpu()
    # give the last convolution full-size weights so that every layer matters
    off = p.numel() - (27 * 16 * 16 + 16)
    g = torch.Generator().manual_seed(seed + 1)
    p[off:off + 27 * 16 * 16] = torch.randn(27 * 16 * 16, generator=g) * (2.0 / (27 * 16)) ** 0.5
    p[p.numel() - 16:] = 0.05 * torch.randn(16, generator=g)
    net.set_params(p)
    x = torch.randn((16, NY, NZ, NX), generator=g, dtype=torch.float64)
    x[15] = 0.0
    x0 = L.to_act(x)
    xb = x.to(torch.bfloat16).double()
    return net, p.double(), x0, xb


def _rel(a, b):
    return float((a.double() - b.double()).norm() / b.double().norm())


def _check_grads(grads, ref_grad):
    import unet_ref
    o = 0
    for cin, cout, _ in unet_ref.SPEC:
        n = 27 * cin * cout + cout
        assert _rel(grads[o:o + n], ref_grad[o:o + n]) < 5e-2, (cin, cout, o)
        o += n


def test_unet_forward_matches_reference():
    import unet_ref
    net, p, x0, xb = _net_and_input(0)
    o = net.forward(x0).cpu()
    ref = unet_ref.forward(p, xb, bf16=True)
    assert _rel(o, ref) < 1e-2
    assert float((o.double() - ref).abs().max()) < 5e-2 * float(ref.abs().max())


def test_unet_gradients_match_reference():
    import unet_ref
    net, p, x0, xb = _net_and_input(1)
    g = torch.Generator().manual_seed(5)
    target = torch.randn((NY, NZ, NX), generator=g, dtype=torch.float64)
    net.zero_grads()
    net.forward(x0)
    loss = net.backward(target.float().cuda())
    grads = net.grads().cpu().double()
    ref_loss, ref_grad, _ = unet_ref.loss_and_grad(p, xb, target, bf16=True)
    assert loss == pytest.approx(ref_loss, rel=2e-2)
    _check_grads(grads, ref_grad)


def test_unet_residual_loss_gradients_match_reference():
    """The residual loss mean((A z - rhat)^2) (A and A^T stencil kernels) and its
    gradients against autograd through the reference's interior stencil."""
    import unet_ref
    net, p, x0, xb = _net_and_input(4)
    g = torch.Generator().manual_seed(9)
    coefs = 0.1 * torch.rand((15, NY, NZ, NX), generator=g, dtype=torch.float64)
    coefs[0] = -(1.0 + torch.rand((NY, NZ, NX), generator=g, dtype=torch.float64))
    coefs = coefs.float().double()
    rhat = torch.randn((NY, NZ, NX), generator=g, dtype=torch.float64).float().double()
    net.zero_grads()
    net.forward(x0)
    loss = net.backward_residual(coefs.float().cuda().contiguous(), rhat.float().cuda().contiguous())
    grads = net.grads().cpu().double()
    ref_loss, ref_grad = unet_ref.residual_loss_and_grad(p, xb, coefs, rhat, bf16=True)
    assert loss == pytest.approx(ref_loss, rel=2e-2)
    _check_grads(grads, ref_grad)


def test_unet_directional_derivative():
    """(L(p + eps d) - L(p - eps d)) / 2 eps from device forward passes agrees with
    <grad L, d> from the device backward pass.  d_i = p_i sign(g_i p_i): a 1-2%
    relative change of every weight, above the BF16 weight rounding; central
    differences at eps and eps/2 are Richardson-extrapolated."""
    net, p, x0, _ = _net_and_input(2)
    g = torch.Generator().manual_seed(6)
    target = torch.randn((NY, NZ, NX), generator=g).cuda()
    net.zero_grads()
    net.forward(x0)
    net.backward(target)
    grad = net.grads().cpu().double()
    d = p * torch.sign(grad * p)

    def loss_at(q):
        net.set_params(q.float())
        net.zero_grads()
        net.forward(x0)
        return net.backward(target)

    def fd(e):
        return (loss_at(p + e * d) - loss_at(p - e * d)) / (2 * e)

    eps = 2e-2
    est = (4.0 * fd(eps / 2) - fd(eps)) / 3.0
    assert est == pytest.approx(float(grad @ d), rel=0.1)


NT = (48, 40, 16)


@pytest.fixture(scope="module")
def trained():
    """A network trained with the residual loss on four terrains (48 x 40 x 16)."""
    from hicar_b200 import learned as L
    net = L.UNet(*NT, seed=3)
    pairs = []
    for s in range(4):
        case = cases.build_case(*NT, seed=100 + s, adv_den=True, n_hills=8)
        pairs += L.training_pairs(case, net, 8, seed=s)
    hist = L.train(net, pairs, steps=400, lr=2e-3, batch=4)
    return net, hist


def test_unet_training_reduces_loss(trained):
    _, hist = trained
    assert np.mean(hist[-20:]) < 0.5 * np.mean(hist[:5])


def test_learned_precond_ab_against_jacobi(trained):
    """Unseen terrain: FGMRES with the learned preconditioner needs fewer
    iterations than FGMRES with the reference Jacobi preconditioner, and both
    reach the same solution (the Jacobi one is checked against the oracle in
    test_gpu_fgmres.py)."""
    from hicar_b200 import learned as L, wind, wind_iterative as wi
    net, _ = trained
    case = cases.build_case(*NT, seed=777, adv_den=True, n_hills=8)
    dom, h = L.calibrated_handle(case)
    net.attach(h)
    div = torch.empty((dom.ny, dom.nz, dom.nx), dtype=torch.float32, device="cuda")
    res = {}
    for name, pc in (("jacobi", _capi.PRECOND_JACOBI), ("learned", _capi.PRECOND_LEARNED)):
        wi.set_options(wi.WindOptions(tol_rel=1e-8, wind_solver_iterations=3000, solver=_capi.SOLVER_FGMRES,
                                      precond=pc))
        dom.set_winds(case.u, case.v, case.w)
        _capi.load().hicarw_reset_solution(h, None)
        wind.calc_divergence(div, dom, use_dqdt=True)
        st = wi.calc_iter_winds(dom, dom.wind_alpha, div, True)
        lam = np.empty((dom.ny + 2, dom.nz + 2, dom.nx + 2))
        _capi.load().hicarw_get_lambda(h, lam.ctypes.data, _capi.MEM_HOST, None)
        res[name] = (st, lam)
    st_j, lam_j = res["jacobi"]
    st_l, lam_l = res["learned"]
    assert st_j["status"] == 0 and st_l["status"] == 0
    assert st_l["precond"] == _capi.PRECOND_LEARNED
    assert st_l["iterations"] < st_j["iterations"]
    assert st_l["true_res"] <= 1.05 * st_l["target"]
    assert np.linalg.norm(lam_l - lam_j) <= 1e-5 * np.linalg.norm(lam_j)
    _capi.check(_capi.load().hicarw_set_learned_precond(h, None), h)
