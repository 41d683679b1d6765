"""Batched and served registrations: every result equals the plain single-pair result for the
same request, bit for bit, whatever else runs beside it; admission respects the HBM budget.

The batch runs every pair of a group through one graph per level whose stages each cover all the
pairs that need them; each pair's arithmetic (walks, reductions and their order, line-search
control) is its plain registration's, so the grids, NMI values and evaluation counts must be
identical, whatever the group size and the gradient-stage scheduling."""
import numpy as np
import pytest

import niftyreg_b200 as nrb
from niftyreg_b200 import phantom
from tests.helpers import ensure_built

pytestmark = pytest.mark.gpu

SHAPES = [(40, 48, 56), (64, 64, 64), (48, 40, 36), (56, 64, 48)]  # (nz, ny, nx), uneven sizes


@pytest.fixture(scope="module")
def pairs():
    ensure_built()
    import torch
    torch.cuda.set_device(0)
    return [phantom.blobs_pair(s, seed=10 + i) for i, s in enumerate(SHAPES)]


def _params():
    return nrb.default_params(levels=2, max_iterations=30, bending_energy=0.005, spacing=(-5.0,),
                              ref_bins=64, flo_bins=64)


@pytest.fixture(scope="module")
def plain(pairs):
    return [nrb.register_host(p.reference, p.floating, p.pixdim, _params()) for p in pairs]


def _same(a, b):
    (ca, ra), (cb, rb) = a, b
    assert np.array_equal(ca, cb)
    assert ra.final_nmi == rb.final_nmi
    assert ra.objective_evaluations == rb.objective_evaluations
    assert ra.gradient_evaluations == rb.gradient_evaluations


def test_batch_equals_plain(pairs, plain):
    out = nrb.register_batch([(p.reference, p.floating, p.pixdim) for p in pairs], _params(), concurrency=4)
    for a, b in zip(out, plain):
        _same(a, b)


@pytest.mark.parametrize("percent,concurrency,group_mb", [(1, 8, 96), (100, 8, 0), (50, 3, 96), (50, 1, 96),
                                                       (50, 8, 1)])
def test_batch_scheduling_changes_nothing(pairs, plain, percent, concurrency, group_mb):
    """The gradient stage run as soon as one pair waits, only when all do, groups of 3 and of 1
    pair, no image cap on a group and a cap that makes every pair a group of its own: the same
    results bit for bit, each at its own index although the batch is grouped by size (the batch
    holds each pair twice, so a group also mixes copies of the same registration)."""
    params = _params()
    params.batch_gradient_percent = percent
    params.batch_group_mb = group_mb
    out = nrb.register_batch([(p.reference, p.floating, p.pixdim) for p in pairs * 2], params,
                             concurrency=concurrency)
    for i, a in enumerate(out):
        _same(a, plain[i % len(pairs)])


def test_batch_budget_for_one_worker(pairs, plain):
    """A budget that holds the largest pair but not in half: the groups run one after another
    on one worker (two workers take half the budget each), with the same results."""
    params = _params()
    big = max(nrb.footprint(p.dim, p.pixdim, params) for p in pairs)
    out = nrb.register_batch([(p.reference, p.floating, p.pixdim) for p in pairs], params, concurrency=4,
                             budget_bytes=int(1.5 * big))
    for a, b in zip(out, plain):
        _same(a, b)
    with pytest.raises(nrb.NrbError, match="larger than the HBM budget"):
        nrb.register_batch([(p.reference, p.floating, p.pixdim) for p in pairs], params, concurrency=4,
                           budget_bytes=big // 2)


def test_batch_without_bending_energy_and_one_level(pairs):
    """No bending-energy stages (weight 0) and a single level, against the plain path."""
    params = nrb.default_params(levels=1, max_iterations=25, bending_energy=0.0, spacing=(-5.0,),
                                ref_bins=32, flo_bins=32)
    want = [nrb.register_host(p.reference, p.floating, p.pixdim, params) for p in pairs[:3]]
    out = nrb.register_batch([(p.reference, p.floating, p.pixdim) for p in pairs[:3]], params, concurrency=3)
    for a, b in zip(out, want):
        _same(a, b)


def test_server_mix_equals_plain(pairs, plain):
    """Requests submitted while others run; each result as when run alone."""
    with nrb.Server(slots=3) as srv:
        tickets = [srv.submit(p.reference, p.floating, p.pixdim, _params()) for p in pairs * 2]
        outs = [srv.wait(t) for t in tickets]
        _, peak_active = srv.stats()
        peak_group = srv.peak_group()
    assert peak_active >= 2 and peak_group >= 2
    for i, (cpp, res, q, lat) in enumerate(outs):
        _same((cpp, res), plain[i % len(pairs)])
        assert lat >= q >= 0.0


def test_server_budget_serialises(pairs, plain):
    """Admission never takes the admitted footprint above the budget; requests that each fill the
    budget run one at a time (groups of one), with the results of the plain path."""
    prm = _params()
    fps = [nrb.footprint(p.dim, p.pixdim, prm) for p in pairs]
    budget = max(fps) + min(fps) // 2
    with nrb.Server(slots=4, budget_bytes=budget) as srv:
        tickets = [srv.submit(p.reference, p.floating, p.pixdim, prm) for p in pairs]
        outs = [srv.wait(t) for t in tickets]
        peak_bytes, _ = srv.stats()
    assert peak_bytes <= budget
    for (cpp, res, _, _), b in zip(outs, plain):
        _same((cpp, res), b)
    big = int(np.argmax(fps))
    with nrb.Server(slots=4, budget_bytes=fps[big]) as srv:
        tickets = [srv.submit(pairs[big].reference, pairs[big].floating, pairs[big].pixdim, prm) for _ in range(3)]
        outs = [srv.wait(t) for t in tickets]
        peak_bytes, peak_active = srv.stats()
        peak_group = srv.peak_group()
    assert peak_bytes <= fps[big] and peak_active == 1 and peak_group == 1
    for cpp, res, _, _ in outs:
        _same((cpp, res), plain[big])


def test_server_rejects_oversized(pairs):
    prm = _params()
    p = pairs[1]
    with nrb.Server(slots=1, budget_bytes=nrb.footprint(p.dim, p.pixdim, prm) - 1) as srv:
        with pytest.raises(nrb.NrbError):
            srv.submit(p.reference, p.floating, p.pixdim, prm)


def test_default_memory_pool_left_alone(pairs):
    """Registrations, batches and servers allocate from the library's own memory pool: the
    application's default pool keeps its release threshold and its reuse setting."""
    import ctypes
    nrb.lib()
    path = next(line.split()[-1] for line in open("/proc/self/maps") if "libcudart" in line)
    rt = ctypes.CDLL(path)

    def settings():
        pool, thr, reuse = ctypes.c_void_p(), ctypes.c_uint64(), ctypes.c_int()
        assert rt.cudaDeviceGetDefaultMemPool(ctypes.byref(pool), 0) == 0
        assert rt.cudaMemPoolGetAttribute(pool, 4, ctypes.byref(thr)) == 0  # release threshold
        assert rt.cudaMemPoolGetAttribute(pool, 3, ctypes.byref(reuse)) == 0  # internal dependencies
        return thr.value, reuse.value

    before = settings()
    p = pairs[0]
    nrb.register_host(p.reference, p.floating, p.pixdim, _params())
    nrb.register_batch([(q.reference, q.floating, q.pixdim) for q in pairs], _params(), concurrency=2)
    with nrb.Server(slots=2) as srv:
        srv.wait(srv.submit(p.reference, p.floating, p.pixdim, _params()))
        assert settings() == before
    assert settings() == before


def test_memory_trim_returns_pool_memory(pairs, plain):
    """After registrations the library's pool keeps what they freed; nrb_memory_trim gives it
    back to the driver, and the next registration maps what it needs again, same result."""
    import torch
    p = pairs[1]
    nrb.register_host(p.reference, p.floating, p.pixdim, _params())
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info()
    nrb.memory_trim(0)
    free_after, _ = torch.cuda.mem_get_info()
    assert free_after > free_before
    _same(nrb.register_host(p.reference, p.floating, p.pixdim, _params()), plain[1])
