"""GPU: the request server.  Each result is the same alone and in the mix
(bit-exact against a plain frsz2_compress / frsz2_decompress of the same
request); admission respects the memory budget; failures are injected on the
host (bad dtype, over-budget, cancelled) and leave the other requests
untouched."""
import ctypes
import os

import numpy as np
import pytest
import torch

import frsz_b200
from frsz_b200 import serve, workloads

pytestmark = pytest.mark.gpu

_cudart = None


def d2h(ptr: int, nbytes: int) -> np.ndarray:
    """Copy raw device memory (a server arena output) to the host."""
    global _cudart
    if _cudart is None:
        cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
        _cudart = ctypes.CDLL(os.path.join(cuda, "lib64", "libcudart.so"))
    out = np.empty(nbytes, dtype=np.uint8)
    assert _cudart.cudaMemcpy(ctypes.c_void_p(out.ctypes.data), ctypes.c_void_p(ptr), ctypes.c_size_t(nbytes), 2) == 0
    return out


def mix(seed, count=40):
    rng = np.random.default_rng(seed)
    reqs = []
    for i in range(count):
        is64 = bool(rng.random() < 0.5)
        dt = np.float64 if is64 else np.float32
        n = int(np.exp(rng.uniform(np.log(10), np.log(3_000_000))))
        bits = int(rng.choice([12, 16, 32]))
        E = int(rng.choice([32, 32, 64, 5]))
        x = torch.from_numpy(workloads.loguniform_np(n, dt, seed=seed * 100 + i, lo=-10, hi=10)).cuda()
        op = serve.OP_COMPRESS if rng.random() < 0.6 else serve.OP_DECOMPRESS
        reqs.append(dict(op=op, dt=dt, is64=is64, bits=bits, E=E, n=n, x=x))
    return reqs


def expected(q):
    if q["op"] == serve.OP_COMPRESS:
        size = frsz_b200.compressed_size(q["dt"], q["bits"], q["E"], q["n"])
        buf = torch.zeros(size, dtype=torch.uint8, device="cuda")
        frsz_b200.compress(q["x"], q["bits"], q["E"], out=buf)
        return buf
    comp = frsz_b200.compress(q["x"], q["bits"], q["E"])
    q["comp"] = comp
    return frsz_b200.decompress(comp, q["n"], q["dt"], q["bits"], q["E"])


def test_results_same_alone_and_in_mix(cuda):
    reqs = mix(1)
    want = [expected(q) for q in reqs]  # each request alone
    torch.cuda.synchronize()
    sv = serve.Server(memory_budget=256 << 20, max_batch=8, streams=3)
    outs, creqs = [], []
    for q in reqs:
        inp = q["x"] if q["op"] == serve.OP_COMPRESS else q["comp"]
        if len(creqs) % 2 == 0:   # half into caller buffers, half into the arena
            o = torch.full_like(want[len(creqs)], 0) if q["op"] == serve.OP_COMPRESS else torch.empty_like(q["x"])
            outs.append(o)
            ptr = o.data_ptr()
        else:
            outs.append(None)
            ptr = None
        creqs.append(serve.request(q["op"], q["is64"], q["bits"], q["E"], q["n"], inp.data_ptr(), ptr))
    first = sv.submit(creqs)
    done = {}
    while len(done) < len(creqs):
        for c in sv.poll(wait_ms=100):
            done[c.id - first] = c
    for i, q in enumerate(reqs):
        c = done[i]
        assert c.status == 0, c
        w = want[i]
        nbytes = w.numel() * w.element_size()
        got = outs[i].view(torch.uint8).cpu().numpy() if outs[i] is not None else d2h(c.output, nbytes)
        if q["op"] == serve.OP_COMPRESS and outs[i] is None:
            # unwritten bytes of the arena buffer are undefined: compare the written layout
            ref = w.cpu().numpy()
            eb = frsz_b200.exponent_size(q["dt"], q["bits"], q["E"], q["n"])
            nb = -(-q["n"] // q["E"])
            wb = frsz_b200.word_bits(q["bits"]) // 8
            assert np.array_equal(got[:nb * wb], ref[:nb * wb]), i
            last = q["n"] - (nb - 1) * q["E"]
            bb = -(-q["E"] * q["bits"] // (8 * wb)) * wb
            keep = (nb - 1) * bb + -(-last * q["bits"] // (8 * wb)) * wb
            assert np.array_equal(got[eb:eb + keep], ref[eb:eb + keep]), i
        else:
            assert np.array_equal(got, w.view(torch.uint8).cpu().numpy()), i
        if c.output_bytes:
            sv.release(c.id)
    st = sv.stats()
    assert st["completed"] == len(reqs) and st["arena_used_bytes"] == 0
    assert st["max_batch"] > 1  # requests were batched together
    sv.close()


def test_budget_admission_and_injected_failures(cuda):
    budget = 8 << 20
    sv = serve.Server(memory_budget=budget, max_batch=4, streams=2)
    x = torch.randn(700_000, device="cuda")  # 2.8 MB fp32 -> ~1.4 MB compressed at 16 bits
    reqs = [serve.request(serve.OP_DECOMPRESS, False, 16, 32, 700_000,
                          frsz_b200.compress(x, 16, 32).data_ptr(), None, flags=serve.RELEASE_ON_COMPLETION)
            for _ in range(30)]
    big = serve.request(serve.OP_DECOMPRESS, False, 16, 32, 4_000_000, x.data_ptr(), None)  # 16 MB > budget
    bad = serve.request(serve.OP_COMPRESS, False, 16, 32, 100, x.data_ptr(), None)
    bad.dtype = 9
    later = serve.request(serve.OP_COMPRESS, False, 16, 32, 1000, x.data_ptr(), None,
                          arrival_ns=serve.now_ns() + 60_000_000_000)
    first = sv.submit(reqs + [big, bad, later])
    sv.cancel(first + 32)
    got = {}
    while len(got) < 33:
        for c in sv.poll(wait_ms=100):
            got[c.id - first] = c
    assert all(got[i].status == 0 for i in range(30))
    assert got[30].status == 2 and got[31].status == 1 and got[32].status == serve.CANCELLED
    st = sv.stats()
    assert st["arena_peak_bytes"] <= budget and st["max_inflight_output_bytes"] <= budget
    assert st["arena_used_bytes"] == 0
    sv.close()


def test_outputs_held_until_release(cuda):
    """With a budget for two outputs, a third request waits until one is
    released."""
    x = torch.randn(1 << 20, device="cuda")
    out_bytes = 4 << 20
    sv = serve.Server(memory_budget=2 * out_bytes, max_batch=4, streams=2)
    comp = frsz_b200.compress(x, 32, 32)
    reqs = [serve.request(serve.OP_DECOMPRESS, False, 32, 32, 1 << 20, comp.data_ptr(), None) for _ in range(3)]
    first = sv.submit(reqs)
    done = []
    for _ in range(50):
        done += sv.poll(wait_ms=20)
        if len(done) >= 2:
            break
    assert len(done) == 2
    assert sv.poll(wait_ms=50) == []  # the third cannot be admitted yet
    sv.release(done[0].id)
    third = []
    for _ in range(50):
        third += sv.poll(wait_ms=20)
        if third:
            break
    assert len(third) == 1 and third[0].status == 0
    y = torch.from_numpy(d2h(third[0].output, out_bytes).view(np.float32))
    assert torch.equal(y, frsz_b200.decompress(comp, 1 << 20, torch.float32, 32, 32).cpu())
    sv.close()
