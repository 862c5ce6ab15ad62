import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libturing_sht.so")


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


HAS_GPU = _has_gpu()


@pytest.fixture(scope="session")
def device():
    if not HAS_GPU:
        pytest.skip("no CUDA device")
    from turing_sphere_b200 import requestShtDevice
    return requestShtDevice(0)


# relative L2 errors measured by the parity tests, printed at the end of the run
_PARITY = []


@pytest.fixture
def parity():
    """parity(name, err, bound): records a measured relative L2 error against
    the f64 oracle, asserts it is within `bound`, and returns it."""
    def record(name, err, bound):
        _PARITY.append((name, float(err), float(bound)))
        assert err <= bound, (name, err, bound)
        return err
    return record


def pytest_terminal_summary(terminalreporter):
    if not _PARITY:
        return
    terminalreporter.write_line("relL2 vs the f64 oracle (measured <= bound):")
    for name, err, bound in _PARITY:
        terminalreporter.write_line(f"  {name}: {err:.2e} <= {bound:.0e}")
