"""The replay adjoint at the differentiable configuration's own size: the 64-sphere scene at 256 x 256,
64 spp, depth 4 (65,538 triangles x 3 albedo channels + 65 material roughnesses).

Checks, as in test_gpu_adjoint.py but at full size: the forward against the oracle (rel. RMSE
<= 1e-3); the gradient against the oracle's CPU replay adjoint; 32 random parameters against central
differences with h = 1e-3 within 1e-2 relative (24 albedo entries by common-random-number renders on
the GPU, 8 roughnesses by the oracle's detached-sampling renders, since roughness moves the sampled
directions and the adjoint holds the sampling fixed); and the backward / forward device-time ratio
at most 3."""
import numpy as np
import pytest

import test_gpu_adjoint as small

pytestmark = pytest.mark.gpu

W = H = 256
SPP, DEPTH = 64, 4
H_FD = 1e-3


@pytest.fixture(scope="module")
def problem(oracle):
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    from axomae_b200 import native, scenes
    s = scenes.spheres_scene(W, H, n_spheres=64, seed=4)
    c = native.Context(0)
    c.upload(s)
    c.build()
    ntri = c.info()["triangles"]
    nmat = len(s["materials"])
    assert ntri == 65538 and nmat == 65
    rng = np.random.default_rng(5)
    alb_t = rng.uniform(0.2, 0.8, (ntri, 3)).astype(np.float32)
    rough_t = rng.uniform(0.1, 0.6, nmat).astype(np.float32)
    alb = np.full((ntri, 3), 0.5, np.float32)
    rough = np.full(nmat, 0.3, np.float32)
    fr = native.make_frame(s, W, H, SPP, DEPTH)
    osc = oracle.OracleScene(s)
    yield dict(s=s, c=c, torch=torch, native=native, ntri=ntri, nmat=nmat, alb_t=alb_t, rough_t=rough_t, alb=alb,
               rough=rough, fr=fr, osc=osc, opt=oracle.options(W, H, SPP, DEPTH))
    c.close()


def _render(P, alb, rough):
    torch = P["torch"]
    a = torch.from_numpy(np.ascontiguousarray(alb)).cuda()
    r = torch.from_numpy(np.ascontiguousarray(rough)).cuda()
    P["c"].set_diff_params(a.data_ptr(), r.data_ptr())
    img = torch.zeros((H, W, 4), dtype=torch.float32, device="cuda")
    st = P["c"].render(P["fr"], film_device_ptr=img.data_ptr())
    out = img.cpu().numpy()
    P["c"].set_diff_params(None, None)
    return out, st


def _backward(P, alb, rough, d_image):
    torch = P["torch"]
    a = torch.from_numpy(np.ascontiguousarray(alb)).cuda()
    r = torch.from_numpy(np.ascontiguousarray(rough)).cuda()
    dI = torch.from_numpy(np.ascontiguousarray(d_image, np.float32)).cuda()
    ga = torch.zeros((P["ntri"], 3), dtype=torch.float32, device="cuda")
    gr = torch.zeros(P["nmat"], dtype=torch.float32, device="cuda")
    P["c"].set_diff_params(a.data_ptr(), r.data_ptr())
    st = P["c"].backward(P["fr"], dI.data_ptr(), ga.data_ptr(), gr.data_ptr())
    P["c"].set_diff_params(None, None)
    return ga.cpu().numpy(), gr.cpu().numpy(), st


@pytest.fixture(scope="module")
def grads(problem):
    P = problem
    T, _ = _render(P, P["alb_t"], P["rough_t"])
    I, fst = _render(P, P["alb"], P["rough"])
    dI = np.zeros_like(I)
    dI[..., :3] = 2.0 * (I[..., :3] - T[..., :3])
    ga, gr, bst = _backward(P, P["alb"], P["rough"], dI)
    return dict(T=T, I=I, dI=dI, ga=ga, gr=gr, fst=fst, bst=bst)


def test_c4_forward_matches_oracle(problem, grads):
    P = problem
    P["osc"].set_diff_params(P["alb"], P["rough"])
    ref, _ = P["osc"].render(P["opt"])
    d = (grads["I"][..., :3].astype(np.float64) - ref[..., :3]) / np.maximum(ref[..., :3], 1e-3)
    assert float(np.sqrt(np.mean(d * d))) <= 1e-3


def test_c4_adjoint_matches_oracle_replay(problem, grads):
    P = problem
    P["osc"].set_diff_params(P["alb"], P["rough"])
    ga, gr = P["osc"].backward(P["opt"], grads["dI"], P["ntri"], P["nmat"])
    assert np.linalg.norm(grads["ga"] - ga) <= 1e-3 * np.linalg.norm(ga)
    assert np.linalg.norm(grads["gr"] - gr) <= 2e-3 * np.linalg.norm(gr)


def test_c4_adjoint_vs_central_differences(problem, grads):
    """32 random parameters: 24 albedo entries of visible triangles (2 of the ground's two large
    triangles, whose gradients dwarf the rest, and 22 of the spheres') and 8 material roughnesses."""
    P = problem
    rng = np.random.default_rng(12)
    ga, gr = grads["ga"], grads["gr"]
    flat = np.abs(ga).reshape(-1)
    spheres = 6 + np.flatnonzero(flat[6:] > 1e-2 * flat[6:].max())  # triangles 0, 1: the ground
    assert spheres.size >= 22
    picks = np.concatenate([rng.choice(6, 2, replace=False), rng.choice(spheres, 22, replace=False)])
    for k in picks:
        t, ch = divmod(int(k), 3)
        ap, am = P["alb"].copy(), P["alb"].copy()
        ap[t, ch] += H_FD
        am[t, ch] -= H_FD
        fd = (small._loss(_render(P, ap, P["rough"])[0], grads["T"]) -
              small._loss(_render(P, am, P["rough"])[0], grads["T"])) / (2 * H_FD)
        assert abs(ga[t, ch] - fd) <= 1e-2 * abs(fd) + 1e-6, (t, ch, ga[t, ch], fd)
    osc = P["osc"]
    osc.set_diff_params(P["alb"], P["rough"])
    for m in rng.choice(P["nmat"], 8, replace=False):
        osc.set_perturbation(2, int(m), 0, H_FD)
        lp = small._loss(osc.render(P["opt"])[0], grads["T"])
        osc.set_perturbation(2, int(m), 0, -H_FD)
        lm = small._loss(osc.render(P["opt"])[0], grads["T"])
        osc.set_perturbation()
        fd = (lp - lm) / (2 * H_FD)
        assert abs(gr[m] - fd) <= 1e-2 * abs(fd) + 1e-4, (m, gr[m], fd)


def test_c4_backward_costs_at_most_three_forwards(problem, grads):
    P = problem
    assert grads["bst"].paths == W * H * SPP
    fwd = min(_render(P, P["alb"], P["rough"])[1].device_ms for _ in range(3))
    bwd = min(_backward(P, P["alb"], P["rough"], grads["dI"])[2].device_ms for _ in range(3))
    print("C4 256^2 64 spp: forward %.2f ms, backward %.2f ms, ratio %.2f" % (fwd, bwd, bwd / fwd))
    assert bwd <= 3.0 * fwd
