"""GPU: this repository's kernels against the reference's own GPU kernels
(frsz::compress_gpu / decompress_gpu, include/frsz2.hpp:1258-1290, built
unmodified into oracle/_ref/libfrsz2_ref_gpu.so, launched with the shapes of
the reference's test) on the same device inputs.  The reference's GPU
compress writes the same bytes as its CPU codec, so its output must equal
ours; both directions must be faster here.  Timings are printed and, when
FRSZ2_RESULTS_DIR is set, written there as JSON."""
import json
import os

import numpy as np
import pytest
import torch

import oracle
import frsz_b200

pytestmark = pytest.mark.gpu

CASES = [  # (name, dtype, n, bits, E)
    ("f32_2p26_b16_e32", torch.float32, 1 << 26, 16, 32),
    ("f64_2p25_b16_e32", torch.float64, 1 << 25, 16, 32),
    ("f64_2p25_b21_e32", torch.float64, 1 << 25, 21, 32),
    ("f64_2p25_b32_e32", torch.float64, 1 << 25, 32, 32),
    ("f64_2p25_b21_e64", torch.float64, 1 << 25, 21, 64),
]


def timed(fn, reps=10):
    fn()
    torch.cuda.synchronize()
    ts = []
    for _ in range(reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        b.synchronize()
        ts.append(a.elapsed_time(b))
    return float(np.median(ts))


@pytest.mark.skipif(not os.path.exists(oracle.REF_GPU_SO), reason="reference GPU kernels not built")
def test_faster_than_reference_gpu_kernels(cuda):
    ref = oracle.ref_gpu_lib()
    results = {}
    for name, dt, n, bits, E in CASES:
        x = torch.randn(n, device="cuda", dtype=dt)
        is64 = int(dt == torch.float64)
        size = frsz_b200.compressed_size(dt, bits, E, n)
        ours = torch.zeros(size + 256, dtype=torch.uint8, device="cuda")  # slack: the reference reads one word past
        theirs = torch.zeros(size + 256, dtype=torch.uint8, device="cuda")
        y = torch.empty_like(x)
        s = torch.cuda.current_stream().cuda_stream
        t_oc = timed(lambda: frsz_b200.compress(x, bits, E, out=ours[:size]))
        t_od = timed(lambda: frsz_b200.decompress(ours[:size], n, dt, bits, E, out=y))
        t_rc = timed(lambda: ref.frsz2ref_gpu(is64, bits, E, 1, x.data_ptr(), n, theirs.data_ptr(), s))
        t_rd = timed(lambda: ref.frsz2ref_gpu(is64, bits, E, 0, theirs.data_ptr(), n, y.data_ptr(), s))
        assert ref.frsz2ref_gpu(is64, bits, E, 1, x.data_ptr(), n, theirs.data_ptr(), s) == 0
        torch.cuda.synchronize()
        assert torch.equal(ours[:size], theirs[:size]), f"{name}: reference GPU compress bytes differ"
        nbytes = n * x.element_size() + (-(-n // E)) * (frsz_b200.word_bits(bits) // 8) * (1 + -(-E * bits // frsz_b200.word_bits(bits)))
        results[name] = {"ours_compress_ms": t_oc, "ours_decompress_ms": t_od, "ref_compress_ms": t_rc,
                         "ref_decompress_ms": t_rd, "ours_compress_gbs": nbytes / t_oc / 1e6,
                         "ours_decompress_gbs": nbytes / t_od / 1e6, "ref_compress_gbs": nbytes / t_rc / 1e6,
                         "ref_decompress_gbs": nbytes / t_rd / 1e6, "speedup_compress": t_rc / t_oc,
                         "speedup_decompress": t_rd / t_od}
        del x, ours, theirs, y
    print(json.dumps(results, indent=1))
    out_dir = os.environ.get("FRSZ2_RESULTS_DIR")
    if out_dir:
        with open(os.path.join(out_dir, "reference_gpu_speed.json"), "w") as f:
            json.dump(results, f, indent=1)
    for name, r in results.items():
        assert r["speedup_compress"] > 1.0 and r["speedup_decompress"] > 1.0, (name, r)
