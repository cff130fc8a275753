"""The frsz2 plugin front end: options, configuration, error codes (CPU) and
the compress / decompress round trip against the oracle (GPU)."""
import numpy as np
import pytest
import torch

import oracle
from frsz_b200 import Frsz2Plugin, workloads


def test_options_and_metadata():
    p = Frsz2Plugin()
    assert p.get_options() == {"frsz2:bits": 32, "frsz2:max_exp_block_size": 32}
    assert p.set_options({"frsz2:bits": 16, "frsz2:max_exp_block_size": 8}) == 0
    assert p.get_options() == {"frsz2:bits": 16, "frsz2:max_exp_block_size": 8}
    assert p.get_configuration()["pressio:thread_safe"] == "multiple"
    assert "Supported values: 2, 4, 8" in p.get_documentation()["frsz2:max_exp_block_size"]
    assert (p.prefix, p.version(), p.patch_version()) == ("frsz2", "0.0.2", 2)
    q = p.clone()
    assert q.get_options() == p.get_options() and q is not p


def test_errors_without_device_work():
    p = Frsz2Plugin()
    rc, out = p.compress(np.zeros(10, dtype=np.int32))
    assert (rc, out, p.error_msg) == (1, None, "unsupported dtype")
    p.set_options({"frsz2:max_exp_block_size": 48})
    assert p.compress(np.zeros(10, dtype=np.float32))[0] == 2
    assert p.error_msg == "Unsupported exponent block size: 48"
    p.set_options({"frsz2:max_exp_block_size": 32, "frsz2:bits": 33})
    assert p.compress(np.zeros(10, dtype=np.float32))[0] == 2
    assert p.error_msg == "Unsupported number of bits: 33"
    assert p.decompress(np.zeros(10, np.uint8), np.zeros(3, dtype=np.int16)) == 1


@pytest.mark.gpu
@pytest.mark.parametrize("dtype,bits,E", [(np.float64, 32, 32), (np.float32, 16, 8), (np.float64, 21, 1024)])
def test_round_trip_host_and_device(cuda, dtype, bits, E):
    p = Frsz2Plugin()
    p.set_options({"frsz2:bits": bits, "frsz2:max_exp_block_size": E})
    x = workloads.loguniform_np(30_001, dtype, seed=bits, lo=-10, hi=10).reshape(30_001)
    rc, comp = p.compress(x)
    assert rc == 0
    ref = oracle.compress(x, bits, E, canary=0)
    assert np.array_equal(comp, ref)
    y = np.empty((30_001,), dtype=dtype)
    assert p.decompress(comp, y) == 0
    assert np.array_equal(y.view(np.uint8), oracle.decompress(ref, x.size, dtype, bits, E).view(np.uint8))
    xd = torch.from_numpy(x).cuda()
    rc, dcomp = p.compress(xd)
    assert rc == 0
    yd = torch.empty_like(xd)
    assert p.decompress(dcomp, yd) == 0
    torch.cuda.synchronize()
    assert torch.equal(yd.cpu(), torch.from_numpy(y))
