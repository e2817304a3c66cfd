"""Test infrastructure only: stands in for the few torch.cuda calls bench.py
makes (device, stream, events, synchronize, tensors on "cuda"), so that
bench.py's main arm can run end to end on the stand-in CUDA runtime
(tests/stub_cudart/stub_cudart.cpp) without a GPU. Import it before bench.py.
Times are meaningless there: the point is the bench's own logic and its line."""
import torch


class _Stream:
    cuda_stream = 0x5EED0  # any non-null handle: the stand-in runtime only uses it as a key


class _Event:
    def __init__(self, enable_timing=False):
        pass

    def record(self, stream=None):
        pass

    def elapsed_time(self, other):
        return 1.0


_tensor = torch.tensor


def _tensor_on_cpu(*args, **kwargs):
    if kwargs.get("device") == "cuda":
        kwargs["device"] = "cpu"
    return _tensor(*args, **kwargs)


torch.cuda.set_device = lambda device: None
torch.cuda.Stream = lambda *args, **kwargs: _Stream()
torch.cuda.set_stream = lambda stream: None
torch.cuda.synchronize = lambda *args, **kwargs: None
torch.cuda.Event = _Event
torch.cuda.get_device_name = lambda *args, **kwargs: "stub sm_100 (no GPU)"
torch.tensor = _tensor_on_cpu
