"""The B200 adjoint (ts_b200_adjoint_*, trottersuzuki_b200.adjoint) against the
CPU FP64 adjoint (oracle/ts_oracle.c tso_adjoint_real / tso_adjoint_imag,
themselves checked against central finite differences in test_oracle_pin.py)
and against central finite differences of the B200 forward pass, in real and
in imaginary time (renormalised every step to the initial norm).

Bar: gradients within 1e-10 of the CPU adjoint (relative to the largest
component) and within 1e-6 of central differences.
"""
import numpy as np
import pytest

import oracle as O
from helpers import desc_from_params

pytestmark = pytest.mark.gpu

DT = 1e-3


def case(N=70, Ny=45, L=8.0, steps=40, g=0.0, lhy=0.0, seed=3):
    lat = O.Lattice(N, L, Ny, None)
    rng = np.random.default_rng(seed)
    X, _ = lat.coordinates()
    psi0 = O.gaussian(lat, 1.0, 1.0, -1.0, 0.2) * np.exp(2j * X)
    V = lat.harmonic(1.0, 1.0) + 0.3 * rng.uniform(-1, 1, lat.shape)
    p = lat.params(DT, False, 1.0, g, lhy, 0.0)
    mask = (X > 0).astype(np.float64)
    return lat, p, psi0, V, mask, steps


def loss_and_seed(lat, psi_t, mask):
    dA = lat.delta_x * lat.delta_y
    return float((np.abs(psi_t) ** 2 * mask).sum() * dA), 2.0 * dA * mask * psi_t


def gpu_run(p, V, psi0, steps, every, lam_fn):
    import torch
    from trottersuzuki_b200.adjoint import AdjointEngine
    eng = AdjointEngine(desc_from_params(p), DT, steps, every)
    dev = torch.device("cuda", 0)
    Vt = torch.tensor(V, dtype=torch.float64, device=dev)
    p0 = torch.tensor(psi0, dtype=torch.complex128, device=dev)
    psi_t = eng.forward(Vt, p0).cpu().numpy()
    lam = torch.tensor(lam_fn(psi_t), dtype=torch.complex128, device=dev)
    gv, gp = eng.backward(lam)
    out = psi_t, gv.cpu().numpy(), gp.cpu().numpy()
    eng.close()
    return out


def rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


@pytest.mark.parametrize("g,lhy,every", [(0.0, 0.0, 0), (0.0, 0.0, 7), (4.0, 0.0, 7),
                                         (4.0, 0.5, 10), (2.0, 0.0, 1)],
                         ids=["inverse", "ckpt_linear", "ckpt_gpe", "ckpt_lhy", "ckpt_every_step"])
def test_adjoint_matches_cpu_adjoint(g, lhy, every):
    lat, p, psi0, V, mask, steps = case(g=g, lhy=lhy)
    tr, ti = O.exp_table(V, DT, False)
    psi_ref = O.evolve(p, psi0, tr, ti, steps)
    psi_t, gv, gp = gpu_run(p, V, psi0, steps, every, lambda pt: loss_and_seed(lat, pt, mask)[1])
    assert np.abs(psi_t - psi_ref).max() <= 1e-10
    _, lam = loss_and_seed(lat, psi_ref, mask)
    gv_ref, gp_ref = O.adjoint_real(p, tr, ti, DT, psi0, steps, lam)
    assert rel(gv, gv_ref) <= 1e-10, rel(gv, gv_ref)
    assert rel(gp, gp_ref) <= 1e-10, rel(gp, gp_ref)


def test_adjoint_matches_finite_differences():
    """Central differences of the B200 forward pass at seeded sites."""
    import torch
    from trottersuzuki_b200.adjoint import AdjointEngine
    lat, p, psi0, V, mask, steps = case(N=64, Ny=64, g=3.0, steps=30)
    dev = torch.device("cuda", 0)
    eng = AdjointEngine(desc_from_params(p), DT, steps, 10)

    def loss(Vh, ph):
        Vt = torch.tensor(Vh, dtype=torch.float64, device=dev)
        p0 = torch.tensor(ph, dtype=torch.complex128, device=dev)
        return loss_and_seed(lat, eng.forward(Vt, p0).cpu().numpy(), mask)[0]

    psi_t, gv, gp = gpu_run(p, V, psi0, steps, 10,
                            lambda pt: loss_and_seed(lat, pt, mask)[1])
    rng = np.random.default_rng(7)
    sites = [(int(y), int(x)) for y, x in zip(rng.integers(20, 44, 8), rng.integers(16, 48, 8))]
    h = 1e-5
    fd_v, fd_r, fd_i = [], [], []
    for y, x in sites:
        e = np.zeros_like(V)
        e[y, x] = h
        fd_v.append((loss(V + e, psi0) - loss(V - e, psi0)) / (2 * h))
        fd_r.append((loss(V, psi0 + e) - loss(V, psi0 - e)) / (2 * h))
        fd_i.append((loss(V, psi0 + 1j * e) - loss(V, psi0 - 1j * e)) / (2 * h))
    ys, xs = zip(*sites)
    assert rel(gv[ys, xs], np.array(fd_v)) <= 1e-6
    assert rel(gp.real[ys, xs], np.array(fd_r)) <= 1e-6
    assert rel(gp.imag[ys, xs], np.array(fd_i)) <= 1e-6
    eng.close()


def test_autograd_function():
    import torch
    import trottersuzuki_b200.adjoint as A
    lat, p, psi0, V, mask, steps = case(g=2.0, steps=25)
    dev = torch.device("cuda", 0)
    eng = A.AdjointEngine(desc_from_params(p), DT, steps, 5)
    Vt = torch.tensor(V, dtype=torch.float64, device=dev, requires_grad=True)
    p0 = torch.tensor(psi0, dtype=torch.complex128, device=dev, requires_grad=True)
    m = torch.tensor(mask, device=dev)
    psi_t = A.evolve(Vt, p0, eng)
    L = (psi_t.abs() ** 2 * m).sum() * (lat.delta_x * lat.delta_y)
    L.backward()
    tr, ti = O.exp_table(V, DT, False)
    psi_ref = O.evolve(p, psi0, tr, ti, steps)
    Lref, lam = loss_and_seed(lat, psi_ref, mask)
    assert abs(L.item() - Lref) <= 1e-12
    gv_ref, gp_ref = O.adjoint_real(p, tr, ti, DT, psi0, steps, lam)
    assert rel(Vt.grad.cpu().numpy(), gv_ref) <= 1e-10
    assert rel(p0.grad.cpu().numpy(), gp_ref) <= 1e-10
    eng.close()


def test_adjoint_rejects_unsupported():
    from trottersuzuki_b200 import B200Error
    from trottersuzuki_b200.adjoint import AdjointEngine
    lat, p, *_ = case(g=3.0)
    with pytest.raises(B200Error):
        AdjointEngine(desc_from_params(p), DT, 10, 0)  # inverse steps need g = 0
    lat2 = O.Lattice(32, 8.0)
    pim = lat2.params(DT, True, 1.0, 0.0, 0.0, 0.0, norm0=1.0)
    with pytest.raises(B200Error):
        AdjointEngine(desc_from_params(pim), DT, 10, 0)  # imaginary time needs checkpoints
    lat3 = O.Lattice(32, 8.0, None, None, True, True)
    pper = lat3.params(DT, True, 1.0, 0.0, 0.0, 0.0, norm0=1.0)
    with pytest.raises(B200Error):
        AdjointEngine(desc_from_params(pper), DT, 10, 5)  # closed tiles only


# ------------------------------------------------------------ imaginary time
def case_imag(N=70, Ny=45, L=8.0, steps=40, g=0.0, lhy=0.0, seed=5):
    lat = O.Lattice(N, L, Ny, None)
    rng = np.random.default_rng(seed)
    X, _ = lat.coordinates()
    psi0 = (O.gaussian(lat, 1.0, 1.0, -1.0, 0.2) * (1 + 0.3 * rng.uniform(-1, 1, lat.shape))
            * np.exp(0.8j * X))
    V = lat.harmonic(1.0, 1.0) + 0.3 * rng.uniform(-1, 1, lat.shape)
    n0 = O.expectations(lat, psi0)["norm2"]
    p = lat.params(DT, True, 1.0, g, lhy, 0.0, norm0=n0)
    mask = (X > 0).astype(np.float64)
    return lat, p, psi0, V, mask, steps


@pytest.mark.parametrize("g,lhy,every", [(0.0, 0.0, 7), (4.0, 0.0, 7), (4.0, 0.5, 10),
                                         (2.0, 0.0, 1), (3.0, 0.0, 40), (3.0, 0.0, 8)],
                         ids=["linear", "gpe", "lhy", "every_step", "one_segment",
                              "graph_segments"])
def test_imag_adjoint_matches_cpu_adjoint(g, lhy, every):
    lat, p, psi0, V, mask, steps = case_imag(g=g, lhy=lhy)
    tr, _ = O.exp_table(V, DT, True)
    psi_ref = O.evolve(p, psi0, tr, np.zeros_like(tr), steps)
    psi_t, gv, gp = gpu_run(p, V, psi0, steps, every, lambda pt: loss_and_seed(lat, pt, mask)[1])
    assert np.abs(psi_t - psi_ref).max() <= 1e-10
    _, lam = loss_and_seed(lat, psi_ref, mask)
    gv_ref, gp_ref = O.adjoint_imag(p, tr, DT, psi0, steps, lam)
    assert rel(gv, gv_ref) <= 1e-10, rel(gv, gv_ref)
    assert rel(gp, gp_ref) <= 1e-10, rel(gp, gp_ref)


def test_imag_adjoint_twice_and_new_norm():
    """Two forward/backward rounds on one engine, the second from a psi0 of
    another norm (norm0 is a launch parameter: the graphs follow it)."""
    lat, p, psi0, V, mask, steps = case_imag(g=3.0, steps=24)
    tr, _ = O.exp_table(V, DT, True)
    import torch
    from trottersuzuki_b200.adjoint import AdjointEngine
    eng = AdjointEngine(desc_from_params(p), DT, steps, 8)
    dev = torch.device("cuda", 0)
    for scale in (1.0, 1.7):
        ps0 = psi0 * scale
        pp = lat.params(DT, True, 1.0, 3.0, 0.0, 0.0, norm0=O.expectations(lat, ps0)["norm2"])
        Vt = torch.tensor(V, dtype=torch.float64, device=dev)
        p0 = torch.tensor(ps0, dtype=torch.complex128, device=dev)
        psi_t = eng.forward(Vt, p0).cpu().numpy()
        psi_ref = O.evolve(pp, ps0, tr, np.zeros_like(tr), steps)
        assert np.abs(psi_t - psi_ref).max() <= 1e-10 * scale
        _, lam = loss_and_seed(lat, psi_ref, mask)
        gv, gp = eng.backward(torch.tensor(lam, dtype=torch.complex128, device=dev))
        gv_ref, gp_ref = O.adjoint_imag(pp, tr, DT, ps0, steps, lam)
        assert rel(gv.cpu().numpy(), gv_ref) <= 1e-10
        assert rel(gp.cpu().numpy(), gp_ref) <= 1e-10
    eng.close()


def test_imag_adjoint_matches_finite_differences():
    """Central differences of the B200 imaginary-time forward pass (norm0
    follows psi0) at seeded sites, GPE, checkpoints every 10 steps."""
    import torch
    from trottersuzuki_b200.adjoint import AdjointEngine
    lat, p, psi0, V, mask, steps = case_imag(N=64, Ny=64, g=3.0, steps=30)
    dev = torch.device("cuda", 0)
    eng = AdjointEngine(desc_from_params(p), DT, steps, 10)

    def loss(Vh, ph):
        Vt = torch.tensor(Vh, dtype=torch.float64, device=dev)
        p0 = torch.tensor(ph, dtype=torch.complex128, device=dev)
        return loss_and_seed(lat, eng.forward(Vt, p0).cpu().numpy(), mask)[0]

    psi_t, gv, gp = gpu_run(p, V, psi0, steps, 10, lambda pt: loss_and_seed(lat, pt, mask)[1])
    rng = np.random.default_rng(9)
    sites = [(int(y), int(x)) for y, x in zip(rng.integers(20, 44, 8), rng.integers(16, 48, 8))]
    h = 1e-5
    fd_v, fd_r, fd_i = [], [], []
    for y, x in sites:
        e = np.zeros_like(V)
        e[y, x] = h
        fd_v.append((loss(V + e, psi0) - loss(V - e, psi0)) / (2 * h))
        fd_r.append((loss(V, psi0 + e) - loss(V, psi0 - e)) / (2 * h))
        fd_i.append((loss(V, psi0 + 1j * e) - loss(V, psi0 - 1j * e)) / (2 * h))
    ys, xs = zip(*sites)
    assert rel(gv[ys, xs], np.array(fd_v)) <= 1e-6
    assert rel(gp.real[ys, xs], np.array(fd_r)) <= 1e-6
    assert rel(gp.imag[ys, xs], np.array(fd_i)) <= 1e-6
    eng.close()


def test_imag_adjoint_512_gpe_matches_cpu_adjoint():
    """512 x 512 imaginary-time GPE (g = 50), 60 steps, checkpoints every 20:
    the full-size lattice of the differentiation configuration."""
    lat = O.Lattice(512, 20.0)
    rng = np.random.default_rng(11)
    X, Y = lat.coordinates()
    psi0 = np.exp(-0.5 * ((X + 3.0) ** 2 + Y ** 2)) * np.exp(2j * X) * (
        1 + 0.01 * rng.uniform(-1, 1, lat.shape))
    V = lat.harmonic(1.0, 1.0) + 0.2 * rng.uniform(-1, 1, lat.shape)
    steps, dt = 60, 1e-4
    p = lat.params(dt, True, 1.0, 50.0, 0.0, 0.0, norm0=O.expectations(lat, psi0)["norm2"])
    mask = (X > 0).astype(np.float64)
    tr, _ = O.exp_table(V, dt, True)
    import torch
    from trottersuzuki_b200.adjoint import AdjointEngine
    dev = torch.device("cuda", 0)
    eng = AdjointEngine(desc_from_params(p), dt, steps, 20)
    psi_t = eng.forward(torch.tensor(V, dtype=torch.float64, device=dev),
                        torch.tensor(psi0, dtype=torch.complex128, device=dev)).cpu().numpy()
    psi_ref = O.evolve(p, psi0, tr, np.zeros_like(tr), steps)
    assert np.abs(psi_t - psi_ref).max() <= 1e-10
    _, lam = loss_and_seed(lat, psi_ref, mask)
    gv, gp = eng.backward(torch.tensor(lam, dtype=torch.complex128, device=dev))
    gv_ref, gp_ref = O.adjoint_imag(p, tr, dt, psi0, steps, lam)
    assert rel(gv.cpu().numpy(), gv_ref) <= 1e-10
    assert rel(gp.cpu().numpy(), gp_ref) <= 1e-10
    eng.close()
