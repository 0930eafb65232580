"""Test configuration: import paths and the `gpu` marker.

CPU tests (`-m "not gpu"`) cover the oracle against the golden fixtures and derived
known-answer tests, the host-side tree/connectivity logic, and that libsrmg.so loads
and exports the declared C ABI.  GPU tests (`-m gpu`) are the parity tests: the CUDA
path, called through the C ABI, against the oracle.
"""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "steamroller.jl_b200"), os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); parity tests of the CUDA path")


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
