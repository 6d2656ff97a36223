import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long CPU-side oracle runs")


@pytest.fixture(scope="session")
def ref_built():
    import oracle

    if not oracle.ref_available("serial"):
        try:
            from oracle import build_ref

            build_ref.build()
        except Exception:  # pragma: no cover - reference sources absent
            pass
    if not oracle.ref_available("serial"):
        pytest.skip("reference CPU build (oracle/_ref) not available on this machine")
    return True
