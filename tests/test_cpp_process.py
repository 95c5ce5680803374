"""The C++ mam4::MicrophysicsProcess (include/mam4b_microphysics.hpp) over
the mam4xx reference containers, built by tests/cpp/build_process_check.py
against the reference headers through the host shim.

CPU: the container -> C-ABI column mapping (every input, tendency and mode
output lands on the right field) and validate(). GPU: the process run
through the reference's own AeroProcess<> wrapper column by column, and
through its batched entry, must give mam4b_step_slab's results bit for
bit (the tendencies are added to zero-filled Tendencies)."""

import ctypes
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "cpp", "_build", "libmam4b_process_check.so")


@pytest.fixture(scope="module")
def harness():
    if not os.path.exists(LIB):
        import sys
        sys.path.insert(0, os.path.join(HERE, "cpp"))
        from build_process_check import build
        if not build():
            pytest.skip("process harness not built (mam4xx tree absent at build)")
    L = ctypes.CDLL(LIB)
    P, I, D = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
    L.mam4b_process_check.argtypes = [I, I, P, P, D, I, P, P, ctypes.c_char_p, I]
    L.mam4b_process_check.restype = I
    L.mam4b_process_check_mapping.argtypes = [I, P, P, P]
    L.mam4b_process_check_mapping.restype = I
    return L


def test_container_mapping_and_validate(harness):
    from mam4xx_b200 import native
    i_f = np.zeros(native.NIN, dtype=np.int32)
    t_f = np.zeros(52, dtype=np.int32)
    m_f = np.zeros(16, dtype=np.int32)
    assert harness.mam4b_process_check_mapping(5, i_f.ctypes.data, t_f.ctypes.data,
                                               m_f.ctypes.data) == 0
    assert list(i_f) == list(range(native.NIN))
    assert list(t_f) == list(range(52))
    # dry diameter, wet diameter, wet density written; aerosol water has no
    # field in mam4::Diagnostics
    assert list(m_f) == list(range(12)) + [-1] * 4


@pytest.mark.gpu
@pytest.mark.parametrize("batched", [0, 1])
def test_process_equals_step_slab(harness, cuda_device, batched):
    import torch
    from mam4xx_b200 import native
    from mam4xx_b200.workloads import make_workload
    w = make_workload("c2", ncol=6, nlev=72, seed=71)
    # valid atmosphere for AeroProcess::validate: the workload's Magnus
    # vapour can be negative in hot cells near the top
    w["in_slab"][3] = np.maximum(w["in_slab"][3], 0.0)
    x = np.ascontiguousarray(w["in_slab"])
    n = x.shape[1]
    tend = np.zeros((52, n))
    mode = np.zeros((12, n))
    err = ctypes.create_string_buffer(256)
    rc = harness.mam4b_process_check(w["ncol"], w["nlev"], x.ctypes.data, w["pblh"].ctypes.data,
                                     w["dt"], batched, tend.ctypes.data, mode.ctypes.data, err,
                                     256)
    assert rc == 0, (rc, err.value)
    xd = torch.from_numpy(x).cuda()
    pb = torch.from_numpy(w["pblh"]).cuda()
    out = torch.empty((native.NOUT, n), dtype=torch.float64, device="cuda")
    ctx = native.Context()
    ctx.step_slab(xd.data_ptr(), pb.data_ptr(), out.data_ptr(), n, w["ncol"], w["nlev"], w["dt"])
    torch.cuda.synchronize()
    ref = out.cpu().numpy()
    ctx.close()
    # tendencies added to zero are the tendencies themselves
    assert np.array_equal(tend, ref[:52])
    assert np.array_equal(mode, ref[52:64])
