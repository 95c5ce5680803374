"""Shared test set-up: markers, in-tree native libraries, helpers."""

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def port_oracle():
    from oracle import build_oracle, pyoracle
    if not os.path.exists(pyoracle.PORT_SO):
        build_oracle.build()
    return pyoracle.PortOracle()


@pytest.fixture(scope="session")
def ref_oracle():
    from oracle import build_oracle, pyoracle
    if not os.path.exists(pyoracle.REF_SO):
        build_oracle.build()
    if not pyoracle.reference_available():
        pytest.skip("reference-compiled oracle not built (mam4xx tree absent)")
    return pyoracle.ReferenceOracle()


@pytest.fixture(scope="session")
def cuda_device():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test run without a CUDA device")
    from mam4xx_b200 import build
    if not os.path.exists(build.LIB):
        build.build_product()
    return torch.device("cuda:0")


def state_rel_err(tend_a, tend_b, in_slab, dt):
    """Error of a tendency in units of the state it changes:
    |a - b| * dt / max(|q_before|, |q_after|), with an absolute floor of
    1e-30 in the state's units. Shapes (52, n)."""
    q0 = np.abs(in_slab[5:57])
    q1 = np.abs(in_slab[5:57] + tend_b * dt)
    scale = np.maximum(np.maximum(q0, q1), 1e-30)
    return np.abs(tend_a - tend_b) * dt / scale
