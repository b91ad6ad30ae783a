# SPDX-License-Identifier: Apache-2.0
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) GPU")
    config.addinivalue_line("markers", "slow: large inputs (minutes on one GPU)")


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Oracle, build
    if not os.path.exists(os.path.join(ROOT, "oracle", "liboracle.so")):
        build()
    return Oracle()


@pytest.fixture(scope="session")
def reference():
    from oracle.oracle import REF_SO, Reference
    if not os.path.exists(REF_SO):
        pytest.skip("oracle/_ref/libbenes_ref.so is not built (reference sources absent)")
    return Reference()


@pytest.fixture(scope="session")
def b200():
    import benes_perm_b200 as bp
    return bp


@pytest.fixture(scope="session")
def gpu(b200):
    if not b200.backend_available():
        pytest.fail("no usable B200 device: the gpu tests need one")
    return b200
