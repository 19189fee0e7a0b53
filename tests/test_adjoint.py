"""The adjoint (FF_adjoint_device and the torch.autograd binding) against
central finite differences of L = Ubar U + sum_i Fbar_i . F_i computed in FP64
by the oracle (the CPU restatement pinned to the reference's outputs) at
perturbed positions and charges. Bar: 1e-6 relative in FP64.
"""
import numpy as np
import pytest
import torch

from msmpb_b200 import systems
from msmpb_b200.autograd import msm_energy_forces
from msmpb_b200.forcefield import ForceField
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

UBAR = 0.7
CASES = {
    # one level: pair sum and top FFT
    "water300": lambda: (*systems.water(100, 14.4, 0), dict(cutoff=8.0, order=6, levels=1,
                                                            top_grid=12)),
    # three levels: restriction, level stencils, prolongation as well
    "water1000_L3": lambda: (*systems.water(333, 21.5, 3), dict(cutoff=8.0, order=6,
                                                               levels=3, top_grid=4)),
}


def loss(o, pos, q, fbar):
    e, f, _ = o.energy(pos, q=q)
    return UBAR * e + float((fbar * f).sum())


def adjoint(ff, pos, q, fbar, reuse=True):
    dev = torch.device("cuda", 0)
    p = torch.from_numpy(pos).to(dev)
    qq = torch.from_numpy(q).to(dev)
    fb = torch.from_numpy(fbar).to(dev)
    st = torch.cuda.current_stream().cuda_stream
    n = len(q)
    f = torch.empty((n, 3), dtype=torch.float64, device=dev)
    e = torch.empty(1, dtype=torch.float64, device=dev)
    ff.energy_device(p.data_ptr(), qq.data_ptr(), f.data_ptr(), 0, e.data_ptr(), st)
    dq = torch.empty(n, dtype=torch.float64, device=dev)
    dr = torch.empty((n, 3), dtype=torch.float64, device=dev)
    ff.adjoint_device(p.data_ptr(), qq.data_ptr(), fb.data_ptr(), UBAR, dq.data_ptr(),
                      dr.data_ptr(), reuse=reuse, stream=st)
    torch.cuda.synchronize()
    return dq.cpu().numpy(), dr.cpu().numpy()


def setup(name, precision="fp64"):
    q, pos, edges, kw = CASES[name]()
    fbar = np.random.default_rng(7).standard_normal((len(q), 3))
    ff = ForceField(q, pos, edges, **kw, precision=precision)
    ff.set_timing(False)
    o = Oracle(q, edges, cutoff=kw["cutoff"], nu=kw["order"], levels=kw["levels"],
               top_grid=kw["top_grid"])
    return q, pos, edges, fbar, ff, o


@pytest.mark.parametrize("name", list(CASES))
def test_adjoint_matches_finite_differences(name):
    q, pos, edges, fbar, ff, o = setup(name)
    dq, dr = adjoint(ff, pos, q, fbar)
    atoms = [0, 7, 41, len(q) - 1]
    h_r, h_q = 1e-5, 1e-5
    fd_r, ad_r, fd_q, ad_q = [], [], [], []
    for k in atoms:
        for a in range(3):
            pp, pm = pos.copy(), pos.copy()
            pp[k, a] += h_r
            pm[k, a] -= h_r
            fd_r.append((loss(o, pp, q, fbar) - loss(o, pm, q, fbar)) / (2 * h_r))
            ad_r.append(dr[k, a])
        qp, qm = q.copy(), q.copy()
        qp[k] += h_q
        qm[k] -= h_q
        fd_q.append((loss(o, pos, qp, fbar) - loss(o, pos, qm, fbar)) / (2 * h_q))
        ad_q.append(dq[k])
    fd_r, ad_r, fd_q, ad_q = map(np.array, (fd_r, ad_r, fd_q, ad_q))
    assert np.linalg.norm(ad_r - fd_r) / np.linalg.norm(fd_r) < 1e-6
    assert np.linalg.norm(ad_q - fd_q) / np.linalg.norm(fd_q) < 1e-6
    ff.close()


def test_reuse_and_recompute_agree():
    q, pos, edges, fbar, ff, o = setup("water1000_L3")
    dq1, dr1 = adjoint(ff, pos, q, fbar, reuse=True)
    dq2, dr2 = adjoint(ff, pos, q, fbar, reuse=False)
    assert np.array_equal(dq1, dq2) and np.array_equal(dr1, dr2)
    ff.close()


def test_mixed_adjoint_close_to_fp64():
    q, pos, edges, fbar, ff, o = setup("water1000_L3")
    dq, dr = adjoint(ff, pos, q, fbar)
    mixed = ForceField(q, pos, edges, cutoff=8.0, order=6, levels=3, top_grid=4,
                       precision="mixed")
    mixed.set_timing(False)
    dqm, drm = adjoint(mixed, pos, q, fbar)
    assert np.linalg.norm(drm - dr) / np.linalg.norm(dr) < 1e-4
    assert np.linalg.norm(dqm - dq) / np.linalg.norm(dq) < 1e-4
    ff.close()
    mixed.close()


def test_autograd_binding():
    q, pos, edges, fbar, ff, o = setup("water300")
    dev = torch.device("cuda", 0)
    p = torch.tensor(pos, device=dev, requires_grad=True)
    qq = torch.tensor(q, device=dev, requires_grad=True)
    fb = torch.tensor(fbar, device=dev)
    u, f = msm_energy_forces(ff, p, qq)
    e_o, f_o, _ = o.energy(pos)
    assert abs(u.item() - e_o) / abs(e_o) < 1e-10
    (UBAR * u + (fb * f).sum()).backward()
    dq, dr = adjoint(ff, pos, q, fbar)
    assert np.allclose(p.grad.cpu().numpy(), dr, rtol=1e-12, atol=1e-12)
    assert np.allclose(qq.grad.cpu().numpy(), dq, rtol=1e-12, atol=1e-12)
    ff.close()


def test_force_matching_water3000():
    """The differentiation workload: 1000 rigid 3-site waters (3,000 atoms,
    cubic 31.04 A box), order 6, cutoff 9 A, automatic grid; the
    force-matching loss L = sum_i |F_i - F_tgt_i|^2 with F_tgt the forces of
    the same system under charges perturbed by N(0, 0.01^2) (seed 4). The
    autograd gradient of L with respect to positions and charges (FP64 form)
    against FP64 central differences (step 1e-5) of the oracle's L on 32
    atoms (96 position and 32 charge components), to 1e-6; the forward
    forces against the oracle's to 1e-10 (code/forcefield1.c:225-231)."""
    q, pos, edges, kw = systems.config("water3000")
    n = len(q)
    rng = np.random.default_rng(4)
    q_tgt = q + rng.normal(0.0, 0.01, n)
    ff = ForceField(q, pos, edges, **kw, precision="fp64")
    ff.set_timing(False)
    o = Oracle(q, edges, cutoff=ff.cutoff, nu=ff.order, levels=ff.levels,
               top_grid=ff.top_grid)
    assert (ff.levels, ff.top_grid) == (1, (27, 27, 27))
    _, f_tgt, _ = o.energy(pos, q=q_tgt)
    _, f_o, _ = o.energy(pos)

    dev = torch.device("cuda", 0)
    p = torch.tensor(pos, device=dev, requires_grad=True)
    qq = torch.tensor(q, device=dev, requires_grad=True)
    u, f = msm_energy_forces(ff, p, qq)
    assert np.sqrt(((f.detach().cpu().numpy() - f_o) ** 2).sum() / (f_o ** 2).sum()) < 1e-10
    lval = ((f - torch.tensor(f_tgt, device=dev)) ** 2).sum()
    lval.backward()
    dr = p.grad.cpu().numpy()
    dq = qq.grad.cpu().numpy()

    def lo(pp, qv):
        _, ff_o, _ = o.energy(pp, q=qv)
        return float(((ff_o - f_tgt) ** 2).sum())

    atoms = np.sort(rng.choice(n, 32, replace=False))
    h = 1e-5
    fd_r, ad_r, fd_q, ad_q = [], [], [], []
    for k in atoms:
        for a in range(3):
            pp, pm = pos.copy(), pos.copy()
            pp[k, a] += h
            pm[k, a] -= h
            fd_r.append((lo(pp, q) - lo(pm, q)) / (2 * h))
            ad_r.append(dr[k, a])
        qp, qm = q.copy(), q.copy()
        qp[k] += h
        qm[k] -= h
        fd_q.append((lo(pos, qp) - lo(pos, qm)) / (2 * h))
        ad_q.append(dq[k])
    fd_r, ad_r, fd_q, ad_q = map(np.array, (fd_r, ad_r, fd_q, ad_q))
    assert np.linalg.norm(ad_r - fd_r) / np.linalg.norm(fd_r) < 1e-6
    assert np.linalg.norm(ad_q - fd_q) / np.linalg.norm(fd_q) < 1e-6
    ff.close()
