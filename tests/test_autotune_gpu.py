"""The walk autotuner: the first registration level of each shape times the objective and
gradient walks over a candidate set (block height, z-chunk, resident blocks) and keeps the
fastest in the process's table. The plan decides which block visits which voxels, never a value,
so every result must be bit-identical with the tuner on or off, and in a batch that takes its
z-chunks from the table."""
import numpy as np
import pytest

import niftyreg_b200 as nrb
from niftyreg_b200 import phantom
from tests.helpers import ensure_built

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pairs():
    ensure_built()
    import torch
    torch.cuda.set_device(0)
    return [phantom.blobs_pair(s, seed=40 + i) for i, s in enumerate([(48, 56, 64), (64, 64, 64)])]


def _params(tune):
    return nrb.default_params(levels=2, max_iterations=25, bending_energy=0.005, spacing=(-5.0,), ref_bins=64,
                              flo_bins=64, autotune=int(tune))


def _same(a, b):
    (ca, ra), (cb, rb) = a, b
    assert np.array_equal(ca, cb)
    assert ra.final_nmi == rb.final_nmi
    assert (ra.objective_evaluations, ra.gradient_evaluations) == (rb.objective_evaluations, rb.gradient_evaluations)


def test_tuned_walks_change_no_result(pairs):
    nrb.autotune_clear()
    p = pairs[0]
    off = nrb.register_host(p.reference, p.floating, p.pixdim, _params(False))
    assert nrb.autotune_entries() == []
    on = nrb.register_host(p.reference, p.floating, p.pixdim, _params(True))
    entries = nrb.autotune_entries()
    assert len(entries) == 2  # one per level shape
    for e in entries:
        print(f"[autotune] {e}")
        assert e["candidates"] >= 8
        assert e["objective"]["us"] <= e["objective"]["model_us"]
        assert e["gradient"]["us"] <= e["gradient"]["model_us"]
    _same(on, off)
    again = nrb.register_host(p.reference, p.floating, p.pixdim, _params(True))
    assert len(nrb.autotune_entries()) == 2  # the table is reused, not re-tuned
    _same(again, off)


def test_batch_with_tuned_chunks_equals_plain(pairs):
    nrb.autotune_clear()
    plain = [nrb.register_host(p.reference, p.floating, p.pixdim, _params(True)) for p in pairs]
    assert len(nrb.autotune_entries()) == 4
    out = nrb.register_batch([(p.reference, p.floating, p.pixdim) for p in pairs], _params(True), concurrency=2)
    for a, b in zip(out, plain):
        _same(a, b)
