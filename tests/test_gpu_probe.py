"""The arithmetic-throughput probe behind the bench's compute roofline:
each kind's chains end where exact FP arithmetic puts them (with b = 1 a
chain a <- a + 0.5 stays exact), and the measured rates are positive and
ordered as the hardware's (packed f32x2 at least the scalar FP32 rate,
FP64 below FP32)."""
import pytest
import torch

from picsar_b200 import _lib, peaks

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind", [0, 1, 2])
def test_probe_chains_exact(cuda, kind):
    blocks, threads, iters = 4, 64, 100
    sink = torch.full((blocks * threads,), -1.0, dtype=torch.float32, device="cuda")
    _lib.call("pxrb_fma_probe", kind, blocks, threads, iters, 1.0, 0.5, sink.data_ptr(),
              torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    # 8 chains starting at 0..7 (kind 1: 16 halves starting at 0..15)
    starts = sum(range(16)) if kind == 1 else sum(range(8))
    nchains = 16 if kind == 1 else 8
    expect = starts + nchains * iters * 0.5
    assert torch.all(sink == expect), (sink[:4], expect)
    assert _lib.query("pxrb_fma_probe_flops", kind, blocks, threads, iters) == \
        blocks * threads * iters * 8 * 2 * (2 if kind == 1 else 1)


def test_probe_rejects_bad_arguments(cuda):
    sink = torch.zeros(64, dtype=torch.float32, device="cuda")
    with pytest.raises(_lib.PicsarB200Error):
        _lib.call("pxrb_fma_probe", 3, 1, 64, 1, 1.0, 0.5, sink.data_ptr(), None)
    with pytest.raises(_lib.PicsarB200Error):
        _lib.call("pxrb_fma_probe", 0, 1, 48, 1, 1.0, 0.5, sink.data_ptr(), None)
    assert _lib.query("pxrb_fma_probe_flops", 5, 1, 32, 1) == -1


def test_measured_peaks_ordered(cuda):
    p = peaks.fma_peaks(iters=256)
    assert p["fp32"] > 0 and p["fp64"] > 0
    assert p["fp32x2"] >= 0.9 * p["fp32"]
    assert p["fp64"] < p["fp32"]
