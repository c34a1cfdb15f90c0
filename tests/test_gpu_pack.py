"""RGBA16F packing on the device, bit for bit the reference viewer's
(examples/viewer/half.hpp: round-to-nearest-even, overflow to infinity,
NaN -> sign | 0x7E00, persistent foam substituted into the displacement
alpha), checked against the oracle restatement that is pinned to the
reference's own pack."""
import numpy as np
import pytest

import oceanlib_b200 as ob
import oracle as O
from oceanlib_b200 import abi
from oceanlib_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _device(cuda_device):
    ob.force_simd_level(None)
    yield


def edge_floats(count: int) -> np.ndarray:
    hi = np.arange(1 << 16, dtype=np.uint32) << 16
    lows = np.array([0, 1, 0x0FFF, 0x1000, 0x1001, 0x3000, 0xFFFF, 0x7FFF], np.uint32)
    bits = (hi[:, None] | lows[None, :]).reshape(-1)
    rng = np.random.default_rng(5)
    bits = np.concatenate([bits, rng.integers(0, 2 ** 32, count, dtype=np.uint64).astype(np.uint32)])
    bits = bits[: len(bits) // 4 * 4]
    return bits.view(np.float32).reshape(-1, 4)


@pytest.mark.parametrize("with_alpha", [False, True])
def test_device_pack_matches_the_reference_pack(with_alpha):
    import torch

    src = edge_floats(1 << 20)
    cells = src.shape[0]
    alpha = np.random.default_rng(9).standard_normal(cells).astype(np.float32) if with_alpha else None
    d_src = torch.from_numpy(src.reshape(-1).copy()).cuda()
    d_alpha = torch.from_numpy(alpha).cuda() if with_alpha else None
    d_out = torch.empty(cells * 4, dtype=torch.int16, device="cuda")
    st = ob.lib().ocean_pack_rgba16(d_src.data_ptr(), d_alpha.data_ptr() if with_alpha else None, cells,
                                    d_out.data_ptr(), None)
    assert st == abi.OCEAN_OK
    torch.cuda.synchronize()
    got = d_out.cpu().numpy().view(np.uint16).reshape(cells, 4)
    assert np.array_equal(got, O.pack_rgba16(src, alpha))


def test_batch_rgba16_frame_is_the_packed_fp32_frame_with_foam_alpha():
    descs = [W.foam_patch_512(seed=s) for s in (7, 8)]
    n = 512
    a = ob.OceanBatch(descs, foam=W.foam_desc())
    b = ob.OceanBatch(descs, foam=W.foam_desc())
    disp = np.empty((2, n, n, 4), np.float32)
    normal = np.empty_like(disp)
    vel = np.empty_like(disp)
    foam = np.empty((2, n, n), np.float32)
    hd = np.empty((2, n, n, 4), np.uint16)
    hn = np.empty_like(hd)
    hv = np.empty_like(hd)
    dt = W.FOAM_DT
    for f in range(1, 4):
        a.update_host([f * dt], dt, disp, normal, vel, foam)
        b.update_host_rgba16([f * dt], dt, hd, hn, hv)
    assert np.array_equal(hd.reshape(-1, 4), O.pack_rgba16(disp, foam))
    assert np.array_equal(hn.reshape(-1, 4), O.pack_rgba16(normal))
    assert np.array_equal(hv.reshape(-1, 4), O.pack_rgba16(vel))
    assert (hd.reshape(-1, 4)[:, 3] != 0).any()  # the foam alpha is not empty
    a.close()
    b.close()
