"""GPU: the batched plan against the oracle, array by array -- mixed float
types, widths (including ones without a persistent kernel), block sizes,
sizes, pointers that force separate launches -- before and after autotuning,
compress and decompress."""
import numpy as np
import pytest
import torch

import oracle
import frsz_b200
from frsz_b200 import BatchArray, BatchPlan, workloads

pytestmark = pytest.mark.gpu


def make_batch(specs, seed=0, canary=0x3D):
    rng = np.random.default_rng(seed)
    arrays, host = [], []
    for k, (dtype, n, bits, E) in enumerate(specs):
        x = workloads.loguniform_np(n, dtype, seed=seed * 1000 + k, lo=-12, hi=12)
        tx = torch.from_numpy(x).cuda()
        size = frsz_b200.compressed_size(dtype, bits, E, n)
        buf = torch.full((size,), canary, dtype=torch.uint8, device="cuda")
        out = torch.full_like(tx, float("nan"))
        arrays.append(BatchArray(values=tx, compressed=buf, bits=bits, block_size=E, decompressed=out))
        host.append(x)
    return arrays, host


def check_batch(arrays, host, canary=0x3D):
    for a, x in zip(arrays, host):
        ref = oracle.compress(x, a.bits, a.block_size, canary=canary)
        assert np.array_equal(a.compressed.cpu().numpy(), ref), (x.dtype, x.size, a.bits, a.block_size)
        y = a.decompressed.cpu().numpy()
        want = oracle.decompress(ref, x.size, x.dtype, a.bits, a.block_size)
        assert np.array_equal(y.view(np.uint8), want.view(np.uint8)), (x.dtype, x.size, a.bits, a.block_size)


SPECS = ([(np.float32, n, b, 32) for n, b in ((1000, 8), (70_001, 12), (4096 * 5, 16), (33, 24), (300_000, 32))] +
         [(np.float64, n, b, 32) for n, b in ((2048 * 3 + 1, 8), (50_000, 12), (1, 16), (90_000, 24), (7777, 32))] +
         [(np.float64, 40_000, 21, 64), (np.float32, 12_345, 21, 128), (np.float64, 20_000, 64, 1024),
          (np.float32, 5_000, 13, 32),    # width with only the default CTA shape
          (np.float64, 10_000, 16, 5),    # block size that is not a power of two
          (np.float32, 9_999, 16, 2),     # block smaller than a lane's values
          (np.float64, 0, 16, 32)])       # empty


def test_batch_matches_oracle(cuda):
    arrays, host = make_batch(SPECS, seed=1)
    plan = BatchPlan(arrays)
    info = plan.info()
    assert info["arrays"] == len(SPECS)
    assert info["separate_launches"] == 2 and info["classes"] >= 10
    plan.compress()
    plan.decompress()
    torch.cuda.synchronize()
    check_batch(arrays, host)
    plan.close()


def test_batch_autotune_and_rerun(cuda):
    arrays, host = make_batch(SPECS[:12], seed=2)
    plan = BatchPlan(arrays)
    ms_c = plan.autotune(compress=True)
    ms_d = plan.autotune(compress=False)
    assert ms_c > 0 and ms_d > 0
    info = plan.info()
    assert info["tuned"] == {"decompress": 1, "compress": 1}
    for a in arrays:  # wipe outputs, run the tuned graphs
        a.compressed.fill_(0x3D)
        a.decompressed.fill_(float("nan"))
    plan.compress()
    plan.decompress()
    torch.cuda.synchronize()
    check_batch(arrays, host)


def test_batch_many_small_arrays(cuda):
    rng = np.random.default_rng(5)
    specs = []
    for _ in range(300):
        dt = np.float32 if rng.random() < 0.5 else np.float64
        specs.append((dt, int(rng.integers(1, 20_000)), int(rng.choice([8, 12, 16, 24, 32])), 32))
    arrays, host = make_batch(specs, seed=3)
    plan = BatchPlan(arrays)
    plan.compress()
    plan.decompress()
    torch.cuda.synchronize()
    check_batch(arrays, host)


def test_batch_direction_checks(cuda):
    x = torch.zeros(100, device="cuda")
    buf = torch.zeros(frsz_b200.compressed_size(np.float32, 16, 32, 100), dtype=torch.uint8, device="cuda")
    plan = BatchPlan([BatchArray(values=x, compressed=buf, bits=16, block_size=32, decompressed=None)])
    plan.compress()
    plan2 = BatchPlan([BatchArray(values=None, compressed=buf, bits=16, block_size=32, decompressed=x)])
    with pytest.raises(frsz_b200.Frsz2Error, match="compress-only|decompress-only"):
        plan2.compress()


def test_batch_rejects_misaligned_pointers(cuda):
    x = torch.zeros(101, dtype=torch.float64, device="cuda")
    buf = torch.zeros(frsz_b200.compressed_size(np.float64, 32, 32, 100) + 8, dtype=torch.uint8, device="cuda")
    with pytest.raises(frsz_b200.Frsz2Error, match="misaligned"):
        BatchPlan([BatchArray(values=x[1:], compressed=buf[2:], bits=32, block_size=32)])


def test_batch_padded_and_unpadded_blocks_in_one_class(cuda):
    """Arrays of one (float type, width) class whose exponent blocks end in pad
    bits (E * bits not a multiple of the word width) next to unpadded ones:
    the persistent kernel picks the padded tile body per array."""
    specs = [(np.float32, 30_001, 21, 8), (np.float32, 20_000, 21, 32), (np.float32, 4096 * 3, 21, 16),
             (np.float64, 10_007, 33, 32), (np.float64, 6_000, 33, 64), (np.float64, 2048 * 2 + 9, 33, 4),
             (np.float64, 9_000, 13, 4), (np.float64, 9_000, 13, 16), (np.float32, 7_000, 13, 8)]
    arrays, host = make_batch(specs, seed=5)
    plan = BatchPlan(arrays)
    info = plan.info()
    assert info["separate_launches"] == 0 and info["persistent_arrays"] == len(specs)
    plan.compress()
    plan.decompress()
    torch.cuda.synchronize()
    check_batch(arrays, host)
    plan.autotune(compress=True)
    plan.autotune(compress=False)
    for a in arrays:
        a.compressed.fill_(0x3D)
        a.decompressed.fill_(float("nan"))
    plan.compress()
    plan.decompress()
    torch.cuda.synchronize()
    check_batch(arrays, host)
    plan.close()


def test_batch_views_off_32_bytes(cuda):
    """Arrays whose values and outputs are views 1-3 elements past a 32-byte
    boundary (element-aligned) run as separate launches inside the plan's
    graph, on the fast kernels' instances for such views; the results equal
    the oracle's."""
    specs = [(np.float32, 3 * 4096 + 17, 16, 32, 1), (np.float64, 2 * 2048 + 5, 21, 64, 3),
             (np.float32, 9_000, 12, 8, 2), (np.float64, 5_000, 40, 16, 1), (np.float32, 4096, 16, 32, 0)]
    arrays, host = [], []
    for k, (dtype, n, bits, E, off) in enumerate(specs):
        x = workloads.loguniform_np(n, dtype, seed=70 + k, lo=-12, hi=12)
        tdt = torch.float32 if dtype == np.float32 else torch.float64
        base = torch.zeros(n + 8, dtype=tdt, device="cuda")
        base[off:off + n] = torch.from_numpy(x).cuda()
        out = torch.full((n + 8,), float("nan"), dtype=tdt, device="cuda")
        buf = torch.full((frsz_b200.compressed_size(dtype, bits, E, n),), 0x3D, dtype=torch.uint8, device="cuda")
        arrays.append(BatchArray(values=base[off:off + n], compressed=buf, bits=bits, block_size=E,
                                 decompressed=out[off:off + n]))
        host.append(x)
    plan = BatchPlan(arrays)
    assert plan.info()["separate_launches"] == 4
    plan.compress()
    plan.decompress()
    torch.cuda.synchronize()
    check_batch(arrays, host)
    plan.close()


@pytest.mark.parametrize("one_cta_per_tile,side_by_side", [(True, False), (True, True), (False, True)])
def test_batch_launch_configurations(cuda, one_cta_per_tile, side_by_side):
    """Every launch configuration gives the oracle's bytes and values: one CTA
    per tile (the tile's array from a per-tile index) and the persistent
    class kernels, classes one after another or side by side."""
    arrays, host = make_batch(SPECS[:12], seed=11)
    plan = BatchPlan(arrays)
    for compress in (True, False):
        plan.configure(compress, shape=0, ctas_per_sm=2, side_by_side=side_by_side,
                       one_cta_per_tile=one_cta_per_tile)
    info = plan.info()
    assert info["one_cta_per_tile"] == {"decompress": int(one_cta_per_tile), "compress": int(one_cta_per_tile)}
    plan.compress()
    plan.decompress()
    torch.cuda.synchronize()
    check_batch(arrays, host)
    with pytest.raises(frsz_b200.Frsz2Error, match="shape 0"):
        plan.configure(True, shape=1, one_cta_per_tile=True)
