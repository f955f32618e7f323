import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


@pytest.fixture(scope="session")
def synth_psp8(tmp_path_factory):
    from lynx_b200 import pseudo
    return pseudo.synthetic_si_psp8(str(tmp_path_factory.mktemp("psp") / "Si_synthetic.psp8"))
