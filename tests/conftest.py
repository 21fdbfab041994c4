import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    # the reference oracle library is built from the reference's sources where they
    # exist (oracle/build_ref.sh finds them: $MIDAPACK_REFERENCE or its default);
    # elsewhere the prebuilt oracle/_ref travels with the tree
    ref_so = os.path.join(ROOT, "oracle", "_ref", "libmidapack_ref.so")
    if not os.path.exists(ref_so):
        subprocess.run([os.path.join(ROOT, "oracle", "build_ref.sh"), "--if-present"], check=False,
                       stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)


@pytest.fixture(scope="session")
def ref_lib():
    from oracle import ref
    if not ref.available():
        pytest.skip("reference oracle library not built")
    return ref


@pytest.fixture(scope="session")
def gpu_ctx():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import midapack_b200 as mb
    return mb.Context(0)
