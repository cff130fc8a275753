"""One array split across ranks by block range: the shard plan and the
all-gather exchange, with 2 and 3 gloo ranks on CPU (the oracle stands in
for the per-rank codec there); on a GPU, the block-range C-ABI entry points,
and 2 gloo ranks (two processes on the one GPU) that each compress their
range with the library's kernels and assemble the whole buffer."""
import os

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import oracle
import frsz_b200
from frsz_b200 import shard, workloads


@pytest.mark.parametrize("dtype,n,bits,E,world", [(np.float32, 100_003, 16, 32, 2), (np.float64, 70_001, 21, 64, 3),
                                                  (np.float64, 9_999, 13, 5, 2), (np.float32, 10, 8, 32, 3)])
def test_shard_plan_covers_written_bytes(dtype, n, bits, E, world):
    nb = -(-n // E)
    ranges, blocks = [], []
    for r in range(world):
        b0, b1 = shard.shard_blocks(n, dtype, bits, E, world, r)
        blocks.append((b0, b1))
        ranges += shard.written_ranges(n, bits, E, b0, b1)
    assert blocks[0][0] == 0 and blocks[-1][1] == nb
    assert all(blocks[i][1] == blocks[i + 1][0] for i in range(world - 1))
    # the union of the ranks' byte ranges is exactly what a whole-array compress writes
    x = workloads.normal_np(n, dtype, 1)
    a = oracle.compress(x, bits, E, canary=0x00)
    b = oracle.compress(x, bits, E, canary=0xFF)
    written = a == b  # unwritten bytes keep the two different canaries
    mask = np.zeros(a.size, dtype=bool)
    for o, l in ranges:
        assert not mask[o:o + l].any(), "ranks overlap"
        mask[o:o + l] = True
    assert np.array_equal(mask, written)


def _rank(rank, world, port, dtype, n, bits, E, q):
    try:
        os.environ["MASTER_ADDR"] = "127.0.0.1"
        os.environ["MASTER_PORT"] = str(port)
        dist.init_process_group("gloo", rank=rank, world_size=world)
        x = workloads.loguniform_np(n, dtype, 7, lo=-20, hi=20)
        buf = torch.zeros(oracle.compressed_bytes(bits, E, n), dtype=torch.uint8)
        b0, b1 = shard.shard_blocks(n, dtype, bits, E, world, rank)
        # this rank's blocks, compressed with the oracle into the whole layout
        full = oracle.compress(x, bits, E, canary=0)
        for o, l in shard.written_ranges(n, bits, E, b0, b1):
            buf[o:o + l] = torch.from_numpy(full[o:o + l].copy())
        shard.all_gather_compressed(buf, n, bits, E, dtype, world, rank)
        q.put((rank, bool(np.array_equal(buf.numpy(), full))))
        dist.destroy_process_group()
    except Exception as e:  # report instead of hanging the parent
        q.put((rank, repr(e)))


@pytest.mark.parametrize("world", [2, 3])
def test_all_gather_assembles_whole_buffer(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + world * 7 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank, args=(r, world, port, np.float64, 50_001, 21, 32, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
    assert all(res[r] is True for r in range(world)), res


@pytest.mark.gpu
@pytest.mark.parametrize("dtype,n,bits,E,world", [(torch.float32, 1_000_003, 16, 32, 3),
                                                  (torch.float64, 500_001, 21, 64, 4),
                                                  (torch.float64, 99_999, 13, 5, 2)])
def test_block_range_entry_points(cuda, dtype, n, bits, E, world):
    g = torch.Generator(device="cuda").manual_seed(3)
    x = torch.randn(n, generator=g, device="cuda", dtype=dtype)
    whole = frsz_b200.compress(x, bits, E, out=torch.zeros(frsz_b200.compressed_size(dtype, bits, E, n),
                                                            dtype=torch.uint8, device="cuda"))
    parts = torch.zeros_like(whole)
    y = torch.zeros_like(x)
    for r in range(world):
        b0, b1 = shard.shard_blocks(n, dtype, bits, E, world, r)
        shard.compress_shard(x[b0 * E:min(n, b1 * E)], n, bits, E, b0, b1, parts)
        shard.decompress_shard(whole, n, dtype, bits, E, b0, b1, y[b0 * E:min(n, b1 * E)])
    torch.cuda.synchronize()
    assert torch.equal(parts, whole)
    assert torch.equal(y, frsz_b200.decompress(whole, n, dtype, bits, E))


def _gpu_rank(rank, world, port, dtype, n, bits, E, q):
    """One rank on cuda:0: compress its block range with the library's
    kernels into the whole array's layout, all-gather the written ranges
    (gloo, host copies), decompress its range from the assembled buffer."""
    try:
        os.environ["MASTER_ADDR"] = "127.0.0.1"
        os.environ["MASTER_PORT"] = str(port)
        dist.init_process_group("gloo", rank=rank, world_size=world)
        torch.cuda.set_device(0)
        x = workloads.loguniform_np(n, dtype, 11, lo=-20, hi=20)
        b0, b1 = shard.shard_blocks(n, dtype, bits, E, world, rank)
        xs = torch.from_numpy(x[b0 * E:min(n, b1 * E)]).cuda()
        dbuf = torch.zeros(oracle.compressed_bytes(bits, E, n), dtype=torch.uint8, device="cuda")
        shard.compress_shard(xs, n, bits, E, b0, b1, dbuf)
        torch.cuda.synchronize()
        hbuf = dbuf.cpu()
        shard.all_gather_compressed(hbuf, n, bits, E, dtype, world, rank)
        full = oracle.compress(x, bits, E, canary=0)
        ok_bytes = bool(np.array_equal(hbuf.numpy(), full))
        ys = torch.empty_like(xs)
        shard.decompress_shard(hbuf.cuda(), n, dtype, bits, E, b0, b1, ys)
        want = oracle.decompress(full, n, dtype, bits, E)[b0 * E:min(n, b1 * E)]
        uint = np.uint64 if dtype == np.float64 else np.uint32
        ok_vals = bool(np.array_equal(ys.cpu().numpy().view(uint), want.view(uint)))
        dist.barrier()
        dist.destroy_process_group()
        q.put((rank, ok_bytes and ok_vals))
    except Exception as e:  # report instead of hanging the parent
        q.put((rank, repr(e)))


@pytest.mark.gpu
@pytest.mark.parametrize("dtype,n,bits,E", [(np.float64, 1_000_003, 21, 32), (np.float32, 777_777, 13, 5)])
def test_gloo_ranks_with_gpu_kernels(cuda, dtype, n, bits, E):
    """World size 2, both ranks on the one GPU: the assembled buffer equals
    the oracle's whole-array buffer byte for byte, and each rank's decoded
    range equals the oracle's values."""
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29700 + bits + os.getpid() % 1000
    procs = [ctx.Process(target=_gpu_rank, args=(r, world, port, dtype, n, bits, E, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=300) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
    assert all(res[r] is True for r in range(world)), res
