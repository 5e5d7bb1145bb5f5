import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the sm_100a library")


@pytest.fixture(scope="session")
def orc():
    import oracle
    return oracle.lib()


@pytest.fixture(scope="session")
def gpu():
    import prism_b200
    return prism_b200.lib()


@pytest.fixture(scope="session")
def ref():
    """The reference's own code compiled here (oracle/_ref/libprism_ref.so), built on first use
    when the reference tree is present; tests that need it are skipped where it is absent."""
    from oracle import ref_build, ref_lib
    if not ref_lib.available():
        try:
            ref_build.build()
        except RuntimeError as e:
            pytest.skip(f"reference build failed: {e}")
    if not ref_lib.available():
        pytest.skip("oracle/_ref/libprism_ref.so is not built and the reference tree is absent")
    return ref_lib
