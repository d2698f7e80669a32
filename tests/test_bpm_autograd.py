"""BPM behind torch.autograd (qoraholo_b200.autograd.BpmModel): its forward equals the reference's
bpm_forward, its backward (the hand-written adjoint sweep with slice checkpointing) equals the
reference's bpm_vjp gradient -- the golden fixture and the reference CPU build at other sizes --
agrees with central finite differences (h = 1e-3), and does not depend on the checkpoint spacing."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import golden, rel_err

pytestmark = pytest.mark.gpu

G = np.array([0.532, 1.337, 1.2, 0.2], np.float32)


@pytest.fixture(scope="module")
def torch(cuda):
    return cuda


def _model(shape, il, every, chunk=0):
    from qoraholo_b200.autograd import BpmModel

    return BpmModel(shape[0], shape[1], il, G, checkpoint_every=every, chunk=chunk)


def _grad(torch, model, ri, g):
    x = torch.from_numpy(ri).cuda().requires_grad_(True)
    y = model(x)
    y.backward(torch.from_numpy(g).cuda())
    torch.cuda.synchronize()
    return y.detach().cpu().numpy(), x.grad.cpu().numpy()


def test_forward_and_vjp_match_the_reference_fixture(torch):
    g = golden("bpm")
    model = _model(g["ri"].shape, g["illum"], every=4)
    y, grad = _grad(torch, model, g["ri"], g["residual"])
    assert rel_err(y - 1, g["forward"] - 1) < 1e-4
    assert rel_err(grad, g["vjp"]) < 1e-4


@pytest.mark.parametrize("every,chunk", [(0, 0), (1, 0), (5, 0), (16, 0), (7, 2)])
def test_checkpoint_spacing_and_chunks_do_not_change_the_gradient(torch, every, chunk):
    g = golden("bpm")
    ref_y, ref_grad = _grad(torch, _model(g["ri"].shape, g["illum"], every=0), g["ri"], g["residual"])
    y, grad = _grad(torch, _model(g["ri"].shape, g["illum"], every=every, chunk=chunk), g["ri"], g["residual"])
    assert np.array_equal(y, ref_y)
    if chunk == 0:
        assert np.array_equal(grad, ref_grad)  # recomputed envelopes are bitwise the stored ones
    else:
        assert rel_err(grad, ref_grad) < 1e-5  # per-chunk partial sums round differently (as the reference)


def test_vjp_matches_the_reference_cpu_build(torch):
    from oracle import qh_oracle as O
    from oracle import refimpl

    if not refimpl.available():
        pytest.skip("reference CPU build (oracle/_ref) not built")
    rng = np.random.default_rng(5)
    nz, n = 20, 32
    il = O.circular_scan(6, 0.9, G)
    ri = (G[1] + 0.03 * rng.random((nz, n, n))).astype(np.float32)
    r = (rng.standard_normal((6, n, n)) + 1j * rng.standard_normal((6, n, n))).astype(np.complex64) * 0.1
    want = refimpl.bpm_vjp(ri - G[1], r, il, G)
    _, grad = _grad(torch, _model((nz, n), il, every=6), ri, r)
    assert rel_err(grad, want) < 1e-4


def test_gradient_matches_central_finite_differences(torch):
    from oracle import qh_oracle as O

    rng = np.random.default_rng(11)
    nz, n = 16, 32
    il = O.circular_scan(5, 0.9, G)
    ri = (G[1] + 0.02 * rng.random((nz, n, n))).astype(np.float32)
    model = _model((nz, n), il, every=4)
    x0 = torch.from_numpy(ri).cuda()
    with torch.no_grad():
        data = model(x0 + 0.01 * torch.rand_like(x0))

    def loss(x):
        y = model(x)
        return 0.5 * (y - data).abs().pow(2).double().sum()

    x = x0.clone().requires_grad_(True)
    loss(x).backward()
    grad = x.grad.double()
    h = 1e-3
    directions = [torch.from_numpy(rng.uniform(-1, 1, (nz, n, n)).astype(np.float32)).cuda() for _ in range(3)]
    e = torch.zeros_like(x0)
    e[nz // 2, n // 2, n // 2 + 1] = 1.0
    directions.append(e)
    with torch.no_grad():
        for v in directions:
            fd = (loss(x0 + h * v) - loss(x0 - h * v)) / (2 * h)
            an = (grad * v.double()).sum()
            assert abs(float(fd - an)) <= 2e-3 * max(abs(float(an)), 1e-6), (float(fd), float(an))


def test_gradient_descent_through_autograd_reduces_the_misfit(torch):
    from oracle import qh_oracle as O

    nz, n = 16, 32
    il = O.circular_scan(7, 0.9, G)
    truth = np.full((nz, n, n), G[1], np.float32)
    truth[5:11, 12:20, 12:20] += 0.02
    model = _model((nz, n), il, every=4)
    with torch.no_grad():
        data = model(torch.from_numpy(truth).cuda())
    x = torch.full((nz, n, n), float(G[1]), device="cuda", requires_grad=True)
    phase = 2 * np.pi / G[0] * G[3]  # screen phase per unit contrast (dz = pixel)
    opt = torch.optim.SGD([x], lr=1.0 / (len(il) * nz * phase * phase))  # 1 / Lipschitz of the summed misfit
    losses = []
    for _ in range(10):
        opt.zero_grad()
        loss = 0.5 * (model(x) - data).abs().pow(2).sum()
        loss.backward()
        opt.step()
        losses.append(loss.item())
    assert all(b <= a for a, b in zip(losses, losses[1:]))
    assert losses[-1] < 0.5 * losses[0]


def test_rejects_wrong_shapes(torch):
    g = golden("bpm")
    model = _model(g["ri"].shape, g["illum"], every=4)
    with pytest.raises(ValueError):
        model(torch.zeros((3, 24, 24), device="cuda"))
    with pytest.raises(TypeError):
        model(torch.zeros(g["ri"].shape, dtype=torch.float64, device="cuda"))
