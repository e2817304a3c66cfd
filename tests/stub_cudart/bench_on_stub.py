"""Test infrastructure only: runs bench.py (arguments passed through) with
torch.cuda stood in by torch_cuda_stub, for CPU tests of the bench on the
stand-in CUDA runtime -- including under torchrun, one process per rank."""
import os
import runpy
import sys

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import torch_cuda_stub  # noqa: E402,F401

sys.argv = ["bench.py"] + sys.argv[1:]
runpy.run_path(os.path.join(os.path.dirname(os.path.abspath(__file__)), "..", "..", "bench.py"), run_name="__main__")
