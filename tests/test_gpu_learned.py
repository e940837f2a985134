"""GPU forward/backward of the learned-guess network against the numpy reference."""
import numpy as np
import pytest
import torch

from oracle import nn_oracle as nno
from b200dft.mole import Mole
from b200dft.molgen import random_molecule
from b200dft.learned import GuessNet, Batch

pytestmark = pytest.mark.gpu


def _mols():
    rng = np.random.default_rng(2)
    return [Mole("C 0 0 0; O 0 0 1.2; H 0.9 0.5 -0.3; H -0.9 0.5 -0.3"), Mole(random_molecule(rng, 3))]


def test_forward_matches_reference(cuda):
    mols = _mols()
    net = GuessNet(seed=0, bf16=False, hl=nno.HL, hr=nno.HR)
    p = nno.init_params(0)
    B = Batch(mols)
    z, y, _ = net.forward(B)
    z, y = z.cpu().numpy(), y.cpu().numpy()
    oz, oy = [], []
    for m in mols:
        a, b = nno.forward(p, m.charges, m.coords)
        oz.append(a); oy.append(b)
    np.testing.assert_allclose(z, np.concatenate(oz), rtol=2e-3, atol=2e-4)
    np.testing.assert_allclose(y, np.concatenate(oy), rtol=2e-3, atol=2e-4)


def test_gradients_match_reference(cuda):
    m = _mols()[0]
    net = GuessNet(seed=0, bf16=False, hl=nno.HL, hr=nno.HR)
    p = nno.init_params(0)
    rng = np.random.default_rng(1)
    Dt = rng.normal(size=(m.nao, m.nao))
    Dt = (Dt + Dt.T) / 2 * 0.1
    B = Batch([m])
    z, y, c = net.forward(B)
    D = torch.zeros(B.n_mat, dtype=torch.float64, device="cuda")
    loss, dz, dy = net.assemble(B, z, y, D, torch.from_numpy(Dt.reshape(-1)).cuda())
    g = net.backward(B, c, dz, dy)
    L0, og = nno.backward(p, m.charges, m.coords, Dt)
    assert abs(loss.item() - L0) < 1e-5 * max(1, abs(L0))
    Dp = nno.assemble(*nno.forward(p, m.charges, m.coords), m.charges, m.coords,
                      *nno.graph(m.charges, m.coords)[3:5])
    np.testing.assert_allclose(D.cpu().numpy().reshape(m.nao, m.nao), Dp, atol=1e-5)
    for name, _ in net.shapes:
        got = net.P(name, grad=True).cpu().numpy()
        ref = og[name]
        scale = max(np.abs(ref).max(), 1e-6)
        assert np.abs(got - ref).max() <= 2e-3 * scale, name


def test_training_reduces_loss(cuda):
    mols = _mols()
    B = Batch(mols)
    rng = np.random.default_rng(3)
    Dt = torch.zeros(B.n_mat, dtype=torch.float64, device="cuda")
    for mi, m in enumerate(mols):
        a = rng.normal(size=(m.nao, m.nao)) * 0.2
        o = int(B.mat_off[mi])
        Dt[o:o + m.nao ** 2] = torch.from_numpy(((a + a.T) / 2).reshape(-1))
    net = GuessNet(seed=1)
    l0 = net.train_step(B, Dt, lr=1e-3).item()
    for _ in range(60):
        l1 = net.train_step(B, Dt, lr=1e-3).item()
    assert l1 < 0.5 * l0


def test_trained_guess_gains_over_minao(cuda):
    """the committed trained network (b200dft/weights/guess_net.npz, made by b200dft.train_guess)
    starts held-out molecules closer to convergence: fewer SCF iterations, same energies"""
    from b200dft.engine import RKSEngine
    from b200dft.molgen import config3_batch
    from b200dft.train_guess import load
    net = load()
    mols = [Mole(s) for s in config3_batch(512, seed=0)]
    res = {}
    for guess in ("minao", "learned"):
        eng = RKSEngine(mols, level=0, precision="mixed", guess=guess, net=net)
        r = eng.run_converged()
        res[guess] = (r["iterations"].cpu().numpy(), r["energy"].cpu().numpy(), r["converged"].cpu().numpy())
        eng.close()
    it0, e0, c0 = res["minao"]
    it1, e1, c1 = res["learned"]
    assert c0.all() and c1.all()
    assert it1.mean() < it0.mean() - 0.3            # measured: 6.83 -> 6.21 on 2048 molecules
    assert np.abs(e1 - e0).max() <= 1e-4             # the plain SCF judges: same converged energies


@pytest.mark.parametrize("shape", [(1000, 512, 288), (37, 10, 512), (300, 128, 32), (513, 257, 129),
                                   (128, 128, 64), (129, 130, 65)])
def test_tensor_core_gemm_matches_bf16_simt(cuda, shape):
    """tcgen05 bf16 product (mode 2) == bf16-rounded SIMT product (same inputs, fp32
    accumulation), with bias, transposed operands and beta accumulation"""
    from b200dft.learned import _lib
    from b200dft._lib import ptr, stream_handle
    import ctypes
    M, N, K = shape
    g = torch.Generator(device="cuda").manual_seed(0)
    A = torch.randn(M, K, device="cuda", generator=g)
    B = torch.randn(K, N, device="cuda", generator=g)
    bias = torch.randn(N, device="cuda", generator=g)
    C0 = torch.randn(M, N, device="cuda", generator=g)
    st = ctypes.c_int(-1)
    assert _lib().b2_nn_gemm_status(1, ctypes.byref(st)) == 0
    out, acc = {}, {}
    for mode in (1, 2):
        C = torch.zeros(M, N, device="cuda")
        assert _lib().b2_nn_gemm(M, N, K, ptr(A), K, 1, ptr(B), N, 1, ptr(C), N, ptr(bias), 0.0, mode,
                                 stream_handle()) == 0
        out[mode] = C
        Cb = C0.clone()
        assert _lib().b2_nn_gemm(M, N, K, ptr(A), K, 1, ptr(B), N, 1, ptr(Cb), N, None, 0.5, mode,
                                 stream_handle()) == 0
        acc[mode] = Cb
    # transposed operands through the strides
    Ct = torch.zeros(N, M, device="cuda")
    assert _lib().b2_nn_gemm(N, M, K, ptr(B), 1, N, ptr(A), 1, K, ptr(Ct), M, None, 0.0, 2, stream_handle()) == 0
    torch.cuda.synchronize()
    assert _lib().b2_nn_gemm_status(1, ctypes.byref(st)) == 0 and st.value == 0
    ref = out[1]
    scale = ref.abs().max().item()
    for mode in (2,):
        assert (out[mode] - ref).abs().max().item() <= 1e-4 * scale
        assert (acc[mode] - acc[1]).abs().max().item() <= 1e-4 * scale
    assert (Ct.T - (ref - bias)).abs().max().item() <= 1e-4 * scale
