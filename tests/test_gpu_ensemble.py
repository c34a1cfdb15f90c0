"""GPU ensembles of uneven N (64 seeded sea states, N from 64 to 1024).

Every ocean must come out bit-identical to the oracle whatever schedule the
autotuner picked (sizes in sequence or concurrently with SM shares)."""
import numpy as np
import pytest

import oceanlib_b200 as ob
import oracle as O
from oceanlib_b200 import workloads as W

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


@pytest.fixture(autouse=True)
def _device(cuda_device):
    ob.force_simd_level(None)
    yield


def test_ensemble_is_bit_exact_per_ocean_under_every_schedule():
    descs = W.ensemble_64()
    sizes = sorted({d.size for d in descs})
    assert sizes == [64, 128, 256, 512, 1024]
    # one ocean of each size, checked against the oracle
    pick = [next(i for i, d in enumerate(descs) if d.size == n) for n in sizes]
    results = {}
    for tune in (False, True):
        ens = ob.OceanEnsemble(descs, autotune=tune)
        if tune:
            assert ens.schedule  # the autotuner reports what it chose
        ens.update(12.5)
        ens.synchronize()
        results[tune] = [ens.read(i) for i in pick]
        ens.close()
    for k, i in enumerate(pick):
        od, on, _ = O.update(descs[i], 12.5)
        for tune in (False, True):
            d, n = results[tune][k]
            assert np.array_equal(bits(d), bits(od)), (descs[i].size, tune)
            assert np.array_equal(bits(n), bits(on)), (descs[i].size, tune)


def test_ensemble_graph_replay_matches_per_call_launches():
    # The frame replayed as one CUDA graph gives the same bits as issuing its
    # calls, frame after frame (times change between replays).
    descs = W.ensemble_64(16)
    a = ob.OceanEnsemble(descs, autotune=False)
    b = ob.OceanEnsemble(descs, autotune=False)
    b.set_graph(False)
    for t in (0.5, 3.25, 100.0):
        a.update(t)
        b.update(t)
    a.synchronize()
    b.synchronize()
    for i in range(len(descs)):
        da, na = a.read(i)
        db, nb = b.read(i)
        assert np.array_equal(bits(da), bits(db)), i
        assert np.array_equal(bits(na), bits(nb)), i
    od, on, _ = O.update(descs[3], 100.0)
    d3, n3 = a.read(3)
    assert np.array_equal(bits(d3), bits(od))
    a.close()
    b.close()


def test_ensemble_rejects_bad_descriptors():
    bad = W.ensemble_64(4)
    bad[2].size = 100
    with pytest.raises(ValueError):
        ob.OceanEnsemble(bad, autotune=False)
