"""Measured arithmetic ceilings of the current GPU (the compute side of the
particle kernel's roofline): FP32, packed f32x2 and FP64 FMA throughput from
the library's probe kernel (pxrb_fma_probe), timed with CUDA events."""
import torch

from . import _lib

_lib.register({
    "pxrb_fma_probe": "I I I I f f p s",
    "pxrb_fma_probe_flops": "=i I I I I",
})

KINDS = {"fp32": 0, "fp32x2": 1, "fp64": 2}


def fma_peak(kind, iters=2048, blocks_per_sm=8, threads=256, repeats=3):
    """Best TFLOP/s of `repeats` timed probe launches (after one warm-up) of
    the given kind ("fp32", "fp32x2", "fp64") on the current device."""
    k = KINDS[kind]
    dev = torch.cuda.current_device()
    blocks = torch.cuda.get_device_properties(dev).multi_processor_count * blocks_per_sm
    sink = torch.empty(blocks * threads, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream()
    flops = _lib.query("pxrb_fma_probe_flops", k, blocks, threads, iters)
    _lib.call("pxrb_fma_probe", k, blocks, threads, iters, 1.0, 0.5, sink.data_ptr(),
              stream.cuda_stream)
    best = 0.0
    for _ in range(repeats):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        _lib.call("pxrb_fma_probe", k, blocks, threads, iters, 1.0, 0.5, sink.data_ptr(),
                  stream.cuda_stream)
        b.record(stream)
        b.synchronize()
        best = max(best, flops / (a.elapsed_time(b) * 1e-3) / 1e12)
    return best


def fma_peaks(**kw):
    """{kind: TFLOP/s} for every probe kind."""
    return {kind: fma_peak(kind, **kw) for kind in KINDS}
