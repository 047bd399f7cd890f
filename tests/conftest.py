"""Test configuration: import paths and the `gpu` marker.

`-m "not gpu"` tests run anywhere (oracle pins against golden fixtures, host
logic, the C ABI's exported symbols).  `-m gpu` tests need an sm_100 device
and call the product through its C ABI.
"""
import os
import sys

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
for sub in ("gpu-spect-pet-sysmat_b200", "oracle"):
    path = os.path.join(ROOT, sub)
    if path not in sys.path:
        sys.path.insert(0, path)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU (B200) and the built CUDA library")
