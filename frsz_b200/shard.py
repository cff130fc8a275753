"""One array split across ranks by block range.

Exponent blocks are independent and every block's exponent slot and words
sit at offsets fixed by the layout (rate is fixed), so ranks that own
disjoint block ranges compress / decompress their part with no exchange
(frsz2_compress_blocks / frsz2_decompress_blocks write the whole array's
layout in place).  Assembling the full compressed buffer on every rank is
the one exchange step, an all-gather of each rank's written byte ranges.
"""
from __future__ import annotations

from typing import List, Optional, Tuple

import torch

from ._lib import check, lib
from . import codec

# values per fast-kernel tile; shard boundaries on whole tiles keep every
# shard on the fast kernels' alignment
_TILE_VALUES = {4: 4096, 8: 2048}


def shard_blocks(n: int, dtype, bits: int, block_size: int, world: int, rank: int) -> Tuple[int, int]:
    """Block range [b0, b1) of `rank`: whole tiles where the block size
    divides the tile, as even as the units allow."""
    es = 8 if codec.dtype_code(dtype) == 1 else 4
    nb = -(-n // block_size)
    tile = _TILE_VALUES[es]
    unit = tile // block_size if (block_size <= tile and tile % block_size == 0) else 1
    units = -(-nb // unit)
    per = -(-units // world)
    b0 = min(nb, rank * per * unit)
    b1 = min(nb, b0 + per * unit)
    return b0, b1


def written_ranges(n: int, bits: int, block_size: int, b0: int, b1: int) -> List[Tuple[int, int]]:
    """(offset, length) byte ranges of the compressed buffer that blocks
    [b0, b1) write: their exponent slots and their words (only the written
    words of a partial last block)."""
    if b1 <= b0:
        return []
    w = codec.word_bits(bits)
    nb = -(-n // block_size)
    eb = codec.exponent_size("float64" if bits > 32 else "float32", bits, block_size, n)
    bb = -(-block_size * bits // w) * (w // 8)
    ranges = [(b0 * (w // 8), (b1 - b0) * (w // 8))]
    words = (b1 - b0) * bb
    if b1 == nb and n % block_size:
        last = n - (nb - 1) * block_size
        words = (b1 - b0 - 1) * bb + (-(-last * bits // w)) * (w // 8)
    ranges.append((eb + b0 * bb, words))
    return ranges


def compress_shard(values: torch.Tensor, n: int, bits: int, block_size: int, b0: int, b1: int,
                   compressed: torch.Tensor, stream=None) -> None:
    """Compress blocks [b0, b1) of an n-value array; `values` holds exactly
    those blocks' values, `compressed` is the whole array's buffer."""
    s = (stream or torch.cuda.current_stream()).cuda_stream
    check(lib().frsz2_compress_blocks(codec.dtype_code(values.dtype), bits, block_size, values.data_ptr(), n, b0,
                                      b1 - b0, compressed.data_ptr(), s))


def decompress_shard(compressed: torch.Tensor, n: int, dtype, bits: int, block_size: int, b0: int, b1: int,
                     values: torch.Tensor, stream=None) -> None:
    s = (stream or torch.cuda.current_stream()).cuda_stream
    check(lib().frsz2_decompress_blocks(codec.dtype_code(dtype), bits, block_size, compressed.data_ptr(), n, b0,
                                        b1 - b0, values.data_ptr(), s))


def all_gather_compressed(compressed: torch.Tensor, n: int, bits: int, block_size: int, dtype, world: int,
                          rank: int, group=None) -> None:
    """Make every rank's `compressed` hold the whole array: each rank
    contributes the byte ranges its blocks wrote (torch.distributed; the
    tensors live where the process group's backend wants them)."""
    import torch.distributed as dist

    mine = [compressed[o:o + l] for o, l in written_ranges(n, bits, block_size,
                                                          *shard_blocks(n, dtype, bits, block_size, world, rank))]
    payload = torch.cat(mine) if mine else compressed[:0]
    sizes = []
    for r in range(world):
        rr = written_ranges(n, bits, block_size, *shard_blocks(n, dtype, bits, block_size, world, r))
        sizes.append(sum(l for _, l in rr))
    cap = max(sizes) if sizes else 0
    send = torch.zeros(cap, dtype=torch.uint8, device=compressed.device)
    send[:payload.numel()] = payload
    recv = [torch.empty(cap, dtype=torch.uint8, device=compressed.device) for _ in range(world)]
    dist.all_gather(recv, send, group=group)
    for r in range(world):
        if r == rank:
            continue
        pos = 0
        for o, l in written_ranges(n, bits, block_size, *shard_blocks(n, dtype, bits, block_size, world, r)):
            compressed[o:o + l] = recv[r][pos:pos + l]
            pos += l
