"""Test configuration.

Marker ``gpu``: needs a CUDA device (the parity tests proper, through the C
ABI).  Everything else runs on CPU: the oracle against the reference and the
golden fixtures, the host-side model/symmetry helpers, and that the C-ABI
library loads and exports every declared symbol.
"""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def _ensure_built():
    lib = os.path.join(ROOT, "qmbcuda_b200", "libqmb_b200.so")
    if not os.path.exists(lib):
        # by path: importing the package would load the missing library
        import importlib.util
        spec = importlib.util.spec_from_file_location(
            "qmbcuda_b200_build", os.path.join(ROOT, "qmbcuda_b200", "build.py"))
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        mod.build()
    orc = os.path.join(ROOT, "oracle", "libqmb_oracle.so")
    if not os.path.exists(orc):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "oracle"], check=True)


_ensure_built()


@pytest.fixture(scope="session")
def has_gpu():
    import qmbcuda_b200 as q
    return q.lib().qmb_device_count() > 0


@pytest.fixture(autouse=True)
def _skip_gpu_without_device(request):
    if request.node.get_closest_marker("gpu") is not None:
        import qmbcuda_b200 as q
        if q.lib().qmb_device_count() == 0:
            pytest.fail("gpu test collected on a host without a CUDA device; run with -m 'not gpu'")
