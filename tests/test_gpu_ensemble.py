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


def _check_against_oracle(ens, descs, t, indices):
    for i in indices:
        od, on, ov = O.update(descs[i], t)
        d, n = ens.read(i)
        assert np.array_equal(bits(d), bits(od)), (descs[i].size, i)
        assert np.array_equal(bits(n), bits(on)), (descs[i].size, i)


def test_one_launch_schedule_is_bit_exact_per_ocean():
    # Config 4's 64 sea states (N from 64 to 1024) with every size's tasks in
    # one persistent launch (N = 1024 over 64 lanes a sequence, single rows):
    # one ocean of each size equals the oracle, per call and per graph replay.
    descs = W.ensemble_64()
    sizes = sorted({d.size for d in descs})
    pick = [next(i for i, d in enumerate(descs) if d.size == n) for n in sizes]
    ens = ob.OceanEnsemble(descs, autotune=False)
    ens.set_schedule(ob.OceanEnsemble.ONE_LAUNCH)
    assert ens.schedule_kind == ob.OceanEnsemble.ONE_LAUNCH
    ens.set_graph(False)
    ens.update(12.5)
    ens.synchronize()
    _check_against_oracle(ens, descs, 12.5, pick)
    ens.set_graph(True)
    for t in (3.0, 47.25):
        ens.update(t)
    ens.synchronize()
    _check_against_oracle(ens, descs, 47.25, pick)
    ens.close()


@pytest.mark.parametrize("velocity", [False, True])
def test_one_launch_schedule_small_sizes_and_velocity(velocity):
    # N = 32 (field pairs, 2 lanes a sequence, 32 rows a task)
    # up to 1024 in one launch, several oceans a size, velocity off and on.
    descs = []
    for k, n in enumerate((32, 64, 128, 256, 512, 1024)):
        for j in range(2):
            descs.append(ob.OceanDesc(size=n, patch_length=20.0 + 3.0 * n, wind_speed=9.0 + k + j,
                                      wind_direction=0.3 * k, choppiness=0.8 + 0.1 * j, seed=100 * k + j,
                                      compute_velocity=velocity))
    ens = ob.OceanEnsemble(descs, autotune=False)
    ens.set_schedule(ob.OceanEnsemble.ONE_LAUNCH)
    ens.update(7.75)
    ens.synchronize()
    for i, d in enumerate(descs):
        od, on, ov = O.update(d, 7.75)
        dd, nn = ens.read(i)
        assert np.array_equal(bits(dd), bits(od)), (d.size, i)
        assert np.array_equal(bits(nn), bits(on)), (d.size, i)
        if velocity:
            db = ens.device_buffers(i)
            v = np.empty((d.size * d.size, 4), np.float32)
            assert ob.lib().ocean_copy_to_host(v.ctypes.data, db.velocity, v.nbytes) == 0
            assert np.array_equal(bits(v), bits(ov)), (d.size, i)
    ens.close()


def test_one_launch_schedule_refused_where_sizes_do_not_qualify():
    descs = [ob.OceanDesc(size=16, seed=1), ob.OceanDesc(size=64, seed=2)]
    ens = ob.OceanEnsemble(descs, autotune=False)
    with pytest.raises(ValueError):
        ens.set_schedule(ob.OceanEnsemble.ONE_LAUNCH)
    ens.set_schedule(ob.OceanEnsemble.SEQUENTIAL)
    assert ens.schedule_kind == ob.OceanEnsemble.SEQUENTIAL
    ens.close()


def test_sharded_ensemble_holds_this_ranks_share():
    # Rank 1 of 2: the router's share of config 4, advanced on this GPU; its
    # oceans are the oracle's.
    from oceanlib_b200 import router

    descs = W.ensemble_64(16)
    sh = router.ShardedEnsemble(descs, rank=1, world=2, autotune=False)
    assert sh.indices == router.assign(descs, 2)[1]
    sh.update(4.5)
    sh.synchronize()
    for local in (0, len(sh.indices) - 1):
        i = sh.indices[local]
        od, on, _ = O.update(descs[i], 4.5)
        d, n = sh.ensemble.read(local)
        assert np.array_equal(bits(d), bits(od)) and np.array_equal(bits(n), bits(on)), i
    sh.close()


def test_tensor_form_ensemble():
    # Config 4's sizes in the tensor-core form: N = 64..512 run on the tensor
    # cores, each ocean bit-identical to a tensor-form batch of its own and
    # within 2e-6 of FP64 per channel; N = 1024, which has no tensor-core
    # engine, runs the exact FP32 form and matches the oracle's bits.
    from oceanlib_b200 import abi

    descs = W.ensemble_64(24)
    sizes = sorted({d.size for d in descs})
    assert 1024 in sizes and 64 in sizes
    ens = ob.OceanEnsemble(descs, autotune=True, form=abi.OCEAN_FFT_TENSOR)
    assert "N=1024" in ens.schedule and "no tensor-core engine" in ens.schedule
    t = 37.5
    ens.update(t)
    ens.synchronize()
    for n in sizes:
        i = next(k for k, d in enumerate(descs) if d.size == n)
        d, nrm = ens.read(i)
        if n == 1024:
            od, on, _ = O.update(descs[i], t)
            assert np.array_equal(bits(d), bits(od)) and np.array_equal(bits(nrm), bits(on))
            continue
        alone = ob.OceanBatch([descs[i]], form=abi.OCEAN_FFT_TENSOR)
        cells = n * n
        ad = np.empty((cells, 4), np.float32)
        an = np.empty_like(ad)
        alone.update_host([t], 0.0, ad, an)
        alone.close()
        assert np.array_equal(bits(d), bits(ad)) and np.array_equal(bits(nrm), bits(an)), n
        if n <= 256:
            ref = O.fp64_frame(descs[i], t)
            for name, got in (("displacement", d), ("normal", nrm)):
                r = ref[name].reshape(cells, 4)
                for c in range(3):
                    rms = np.sqrt(np.mean(r[:, c] ** 2))
                    err = np.abs(got.reshape(cells, 4)[:, c].astype(np.float64) - r[:, c]).max() / rms
                    assert err <= 2e-6, (n, name, c, err)
    ens.close()
