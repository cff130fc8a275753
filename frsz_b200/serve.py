"""Request server over the C ABI's frsz2_server_* (continuous batching under
a device-memory budget; see include/frsz2_b200.h).  No counterpart in the
reference."""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import List, Optional, Sequence

from ._lib import FRSZ2_DOUBLE, FRSZ2_FLOAT, CompletionC, CountersC, RequestC, check, lib

OP_COMPRESS = 0
OP_DECOMPRESS = 1
RELEASE_ON_COMPLETION = 1
ARRIVAL_RELATIVE = 2
CANCELLED = 3


def now_ns() -> int:
    return lib().frsz2_now_ns()


@dataclass
class Completion:
    id: int
    status: int
    op: int
    output: int
    output_bytes: int
    bytes: int
    arrival_ns: int
    admit_ns: int
    done_ns: int

    @property
    def latency_ns(self) -> int:
        return self.done_ns - self.arrival_ns


def request(op: int, dtype_is_f64: bool, bits: int, block_size: int, n: int, input_ptr: int,
            output_ptr: Optional[int] = None, arrival_ns: int = 0, flags: int = 0) -> RequestC:
    r = RequestC()
    r.op, r.dtype, r.bits, r.block_size, r.n = op, FRSZ2_DOUBLE if dtype_is_f64 else FRSZ2_FLOAT, bits, block_size, n
    r.input, r.output, r.arrival_ns, r.flags = input_ptr, output_ptr, arrival_ns, flags
    return r


class Server:
    def __init__(self, memory_budget: int, max_batch: int = 256, streams: int = 4):
        h = ctypes.c_void_p()
        check(lib().frsz2_server_create(memory_budget, max_batch, streams, ctypes.byref(h)))
        self._h = h
        self._buf = (CompletionC * 4096)()

    def submit(self, requests: Sequence[RequestC]) -> int:
        arr = (RequestC * len(requests))(*requests) if not isinstance(requests, ctypes.Array) else requests
        first = ctypes.c_uint64()
        check(lib().frsz2_server_submit(self._h, arr, len(requests), ctypes.byref(first)))
        return first.value

    def poll(self, wait_ms: int = 0) -> List[Completion]:
        cnt = ctypes.c_uint64()
        check(lib().frsz2_server_poll(self._h, self._buf, len(self._buf), ctypes.byref(cnt), wait_ms))
        out = []
        for i in range(cnt.value):
            c = self._buf[i]
            out.append(Completion(c.id, c.status, c.op, c.output or 0, c.output_bytes, c.bytes, c.arrival_ns,
                                  c.admit_ns, c.done_ns))
        return out

    def release(self, rid: int) -> None:
        check(lib().frsz2_server_release(self._h, rid))

    def cancel(self, rid: int) -> None:
        check(lib().frsz2_server_cancel(self._h, rid))

    def stats(self) -> dict:
        st = CountersC()
        check(lib().frsz2_server_stats(self._h, ctypes.byref(st)))
        return {k: getattr(st, k) for k, _ in CountersC._fields_}

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().frsz2_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
