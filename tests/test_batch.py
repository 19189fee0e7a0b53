"""Batches (FF_batch_*): many independent systems of uneven size, order and
precision evaluated by one CUDA graph launch.

A member's results in a batch come from the same kernels on the same inputs
as its own FF_energy_device call, so they must be bit-identical to it; the
small members are also checked against the oracle (FP64 members to 1e-10,
mixed members to the FP32 level). Argument checks run without a GPU.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from msmpb_b200 import _lib as L
from msmpb_b200 import systems
from msmpb_b200.forcefield import Batch, ForceField, MSMError

DEV = torch.device("cuda", 0)


def small_batch(count=10, seed=11, precisions=("mixed", "fp64")):
    """Ion boxes of 500..3000 atoms, orders 4/6/8, alternating precision."""
    out = []
    for i, (q, pos, edges, kw) in enumerate(
            systems.ion_batch(count, seed=seed, n_min=500, n_max=3000)):
        ff = ForceField(q, pos, edges, **kw, precision=precisions[i % len(precisions)])
        ff.set_timing(False)
        out.append((q, pos, edges, ff))
    return out


class Buffers:
    """Device inputs and outputs of every member."""

    def __init__(self, members):
        self.pos = [torch.tensor(p, device=DEV) for _, p, _, _ in members]
        self.q = [torch.tensor(q, device=DEV) for q, _, _, _ in members]
        self.f = [torch.full((len(q), 3), np.nan, dtype=torch.float64, device=DEV)
                  for q, _, _, _ in members]
        self.phi = [torch.full((len(q),), np.nan, dtype=torch.float64, device=DEV)
                    for q, _, _, _ in members]
        self.e = torch.full((len(members),), np.nan, dtype=torch.float64, device=DEV)

    def run(self, batch, weights=None):
        st = torch.cuda.current_stream().cuda_stream
        batch.energy_device([t.data_ptr() for t in self.pos], [t.data_ptr() for t in self.q],
                            [t.data_ptr() for t in self.f], [t.data_ptr() for t in self.phi],
                            self.e.data_ptr(), st, weights=weights)
        torch.cuda.synchronize()
        return (self.e.cpu().numpy(), [t.cpu().numpy() for t in self.f],
                [t.cpu().numpy() for t in self.phi])


def single(ff, pos, q, weights=None):
    """The member's own FF_energy_device evaluation."""
    p = torch.tensor(pos, device=DEV)
    qq = torch.tensor(q, device=DEV)
    f = torch.empty((len(q), 3), dtype=torch.float64, device=DEV)
    phi = torch.empty(len(q), dtype=torch.float64, device=DEV)
    e = torch.empty(1, dtype=torch.float64, device=DEV)
    ff.energy_device(p.data_ptr(), qq.data_ptr(), f.data_ptr(), phi.data_ptr(), e.data_ptr(),
                     torch.cuda.current_stream().cuda_stream, weights=weights)
    torch.cuda.synchronize()
    return e.item(), f.cpu().numpy(), phi.cpu().numpy()


def assert_same_as_single(members, e, f, phi, weights=None):
    for i, (q, pos, _, ff) in enumerate(members):
        w = None if weights is None else weights[i]
        e1, f1, p1 = single(ff, pos, q, w)
        assert e[i] == e1, i
        assert np.array_equal(f[i], f1), i
        assert np.array_equal(phi[i], p1), i


@pytest.mark.gpu
@pytest.mark.parametrize("branches", [0, 1, 3, Batch.MERGED, -3])
def test_batch_matches_members(branches):
    members = small_batch()
    b = Batch([m[3] for m in members], branches=branches)
    buf = Buffers(members)
    e, f, phi = buf.run(b)
    if branches:
        assert b.branches() == branches
    else:
        assert -4 <= b.branches() <= len(members) and b.branches() != 0
    if b.branches() < 0:
        # one launch per kernel of each (order, precision) group's sequence
        groups = len({(m[3].order, m[3].struct.precision) for m in members})
        assert b.kernel_launches() <= -b.branches() * groups * max(
            m[3].kernel_launches() for m in members)
        assert b.kernel_launches() < sum(m[3].kernel_launches() for m in members)
    else:
        assert b.kernel_launches() == sum(m[3].kernel_launches() for m in members)
    assert_same_as_single(members, e, f, phi)
    b.close()


@pytest.mark.gpu
def test_merged_batch_levels_and_pme():
    """Merged launches over members of several kinds: one to four levels
    (level stencils, transfers and the top FFT merged), both precisions and
    a triclinic box."""
    members = []
    for i, (q, pos, edges, kw) in enumerate(
            systems.ion_batch(6, seed=21, n_min=800, n_max=2500)):
        kw = dict(kw)
        kw["levels"] = 1 + i % 4
        kw["top_grid"] = 6 if i % 4 else 0
        if not kw["top_grid"]:
            kw.pop("top_grid")
        ff = ForceField(q, pos, edges, **kw, precision=("mixed", "fp64")[i % 2])
        ff.set_timing(False)
        members.append((q, pos, edges, ff))
    q, pos, edges, kw = systems.ion_batch(1, seed=22, n_min=900, n_max=900)[0]
    tri = edges.copy()
    tri[0, 1] = 0.2 * edges[0, 0]
    ff = ForceField(q, pos, tri, **kw, precision="mixed")
    ff.set_timing(False)
    members.append((q, pos, tri, ff))
    b = Batch([m[3] for m in members], branches=Batch.MERGED)
    buf = Buffers(members)
    e, f, phi = buf.run(b)
    assert b.branches() == Batch.MERGED
    assert b.kernel_launches() < sum(m[3].kernel_launches() for m in members)
    assert_same_as_single(members, e, f, phi)
    # replays after new weights and a device box change stay bit-identical
    weights = [[0.75] * (m[3].levels + 1) for m in members]
    e, f, phi = buf.run(b, weights=weights)
    assert_same_as_single(members, e, f, phi, weights)
    members[0][3].rebuild_device(members[0][2] * 0.98, torch.cuda.current_stream().cuda_stream)
    e, f, phi = buf.run(b, weights=weights)
    assert_same_as_single(members, e, f, phi, weights)
    b.close()


@pytest.mark.gpu
def test_batch_against_oracle():
    from oracle.oracle import Oracle
    members = small_batch(count=4, seed=12)
    b = Batch([m[3] for m in members], branches=2)
    e, f, phi = Buffers(members).run(b)
    for i, (q, pos, edges, ff) in enumerate(members):
        o = Oracle(q, edges, cutoff=ff.cutoff, nu=ff.order, levels=ff.levels,
                   top_grid=ff.top_grid)
        eo, fo, _ = o.energy(pos)
        tol_e, tol_f = (1e-11, 1e-10) if i % 2 else (1e-5, 1e-4)
        assert abs(e[i] - eo) / abs(eo) < tol_e, i
        assert np.sqrt(((f[i] - fo) ** 2).sum() / (fo ** 2).sum()) < tol_f, i
        # potentials: U = 1/2 sum q phi
        assert abs(0.5 * q @ phi[i] - e[i]) / abs(e[i]) < tol_e * 10, i
    b.close()


@pytest.mark.gpu
def test_merged_batch_fallback_kernels(monkeypatch):
    """The forms chosen for geometries the default kernels do not take (one
    thread per atom for the pair sum, the slab-staged anterpolation, the
    unfolded level stencils), forced everywhere, through merged launches:
    bit-identical to each member's own evaluation."""
    for var, val in (("MSMPB_PAIR", "thread"), ("MSMPB_ANTERP", "gather"),
                     ("MSMPB_STENCIL", "full")):
        monkeypatch.setenv(var, val)
    members = []
    for i, (q, pos, edges, kw) in enumerate(
            systems.ion_batch(4, seed=23, n_min=800, n_max=2000)):
        kw = dict(kw, levels=1 + i % 3)
        if i % 3:
            kw["top_grid"] = 6
        ff = ForceField(q, pos, edges, **kw, precision=("mixed", "fp64")[i % 2])
        ff.set_timing(False)
        members.append((q, pos, edges, ff))
    b = Batch([m[3] for m in members], branches=Batch.MERGED)
    e, f, phi = Buffers(members).run(b)
    assert b.branches() == Batch.MERGED
    assert_same_as_single(members, e, f, phi)
    b.close()


@pytest.mark.gpu
@pytest.mark.parametrize("branches", [2, Batch.MERGED])
def test_batch_recaptures_on_change(branches):
    members = small_batch(count=6, seed=13)
    b = Batch([m[3] for m in members], branches=branches)
    buf = Buffers(members)
    buf.run(b)
    # new output buffers: the graph is captured again
    buf2 = Buffers(members)
    e, f, phi = buf2.run(b)
    assert_same_as_single(members, e, f, phi)
    # per-member weights (levels + 1 entries each)
    weights = [None] * len(members)
    weights[1] = [0.5] * (members[1][3].levels + 1)
    e, f, phi = buf2.run(b, weights=weights)
    assert_same_as_single(members, e, f, phi, weights)
    # a member's box changes on the device: the next replay uses the new box
    q, pos, edges, ff = members[2]
    ff.rebuild_device(edges * 1.01, torch.cuda.current_stream().cuda_stream)
    e, f, phi = buf2.run(b)
    assert_same_as_single(members, e, f, phi)
    twin = ForceField(q, pos, edges, cutoff=ff.cutoff, order=ff.order, levels=ff.levels,
                      top_grid=ff.top_grid, precision="mixed")
    twin.rebuild(edges * 1.01, pos)
    e2, _, _ = single(twin, pos, q)
    assert abs(e[2] - e2) <= 1e-6 * abs(e2)
    b.close()


@pytest.mark.gpu
def test_batch_recaptures_after_member_engine_replaced():
    """FF_set_precision (like a second FF_build or FF_set_device) replaces a
    member's device engine and frees the old one's buffers: the next batch
    call must capture again rather than replay nodes that point into the
    freed engine."""
    members = small_batch(count=4, seed=15)
    b = Batch([m[3] for m in members], branches=Batch.MERGED)
    buf = Buffers(members)
    buf.run(b)
    members[1][3].set_precision("fp64")
    members[1][3].set_timing(False)
    members[2][3].set_precision("mixed")
    members[2][3].set_timing(False)
    e, f, phi = buf.run(b)
    assert_same_as_single(members, e, f, phi)
    b.close()


@pytest.mark.gpu
def test_batch_rejects_repeated_member():
    members = small_batch(count=2, seed=14)
    with pytest.raises(MSMError) as ex:
        Batch([members[0][3], members[0][3]])
    assert ex.value.code == L.ERR_ARGUMENT


def test_batch_new_argument_checks():
    lib = L.load()
    st = C.c_int(-1)
    assert not lib.FF_batch_new(None, 3, 0, C.byref(st))
    assert st.value == L.ERR_ARGUMENT
    q, pos, edges = systems.ions(500, 0.1, 2.0, 1)
    ff = ForceField(q, pos, edges, order=4, cutoff=8.0)
    arr = (C.POINTER(L.FFStruct) * 1)(ff.ff)
    assert not lib.FF_batch_new(arr, 1, 65, C.byref(st))
    assert st.value == L.ERR_ARGUMENT
    assert not lib.FF_batch_new(arr, 1, -65, C.byref(st))
    assert st.value == L.ERR_ARGUMENT
    if not torch.cuda.is_available():  # built on the host, no device plan
        assert not lib.FF_batch_new(arr, 1, 0, C.byref(st))
        assert st.value == L.ERR_STATE
    assert lib.FF_batch_branches(None) == 0
    assert lib.FF_batch_last_error(None) == L.ERR_ARGUMENT
    lib.FF_batch_delete(None)
    ff.close()


def test_ion_generator():
    from scipy.spatial import cKDTree
    for n in (500, 730, 4000):
        q, pos, edges = systems.ions(n, 0.1, 2.0, 3)
        edge = edges[0, 0]
        assert abs(n / edge ** 3 - 0.1) < 1e-12
        assert q.sum() == 0 and set(np.unique(q)) == {-1.0, 1.0}
        assert pos.min() >= 0 and pos.max() < edge
        d, _ = cKDTree(pos, boxsize=edge).query(pos, k=2)
        assert d[:, 1].min() >= 2.0
    batch = systems.ion_batch(count=6, seed=5, n_max=2000)
    assert [kw["order"] for *_, kw in batch] == [4, 6, 8, 4, 6, 8]
    assert all(500 <= len(b[0]) <= 2000 and len(b[0]) % 2 == 0 for b in batch)
