import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "gpu_pending: needs a CUDA device; written, not yet run on a B200 "
                                       "(run with -m gpu_pending; joins the gpu set once it has passed there)")
    # the reference oracle library is built from /root/reference where that exists;
    # elsewhere (the GPU box) the prebuilt oracle/_ref travels with the tree
    ref_so = os.path.join(ROOT, "oracle", "_ref", "libmidapack_ref.so")
    if not os.path.exists(ref_so) and os.path.isdir("/root/reference/algebra"):
        subprocess.run([os.path.join(ROOT, "oracle", "build_ref.sh")], check=False,
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
