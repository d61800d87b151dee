"""The per-point FLOP count the roofline uses (bench.qp_flops) against the
oracle's counting build: every floating-point operation of the quadrature-point
physics in the oracle's operation order (ORC_COUNT_FLOPS), for beams of 5 to 21
nodes.  CPU only."""
import ctypes
import os

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def counting_oracle():
    from oracle import oracle_py
    oracle_py.build()
    lib = ctypes.CDLL(os.path.join(ROOT, "oracle", "_build", "libkyn_oracle_flops.so"))
    lib.orc_model_create.restype = ctypes.c_void_p
    lib.orc_model_create.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int]
    lib.orc_model_destroy.argtypes = [ctypes.c_void_p]
    lib.orc_predict_and_assemble.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    lib.orc_flops_read.restype = ctypes.c_longlong
    lib.orc_flops_read.argtypes = [ctypes.c_int]
    return lib


@pytest.mark.parametrize("nodes", [5, 8, 13, 17, 21])
def test_quadrature_point_flops(counting_oracle, nodes):
    import bench
    from openturbine_b200 import workloads as W
    L = counting_oracle
    pm = W.batch_cantilever_model(W.BeamDraw(0, nodes, 40.0, 1e4, 1.0)).pack()
    err = ctypes.create_string_buffer(256)
    h = L.orc_model_create(ctypes.byref(pm.desc), err, 256)
    assert h, err.value
    L.orc_flops_reset()
    c = W.batch_params().to_c()
    L.orc_predict_and_assemble(ctypes.c_void_p(h), ctypes.byref(c))
    per_point = L.orc_flops_read(1) / (nodes + 2)
    L.orc_model_destroy(ctypes.c_void_p(h))
    assert per_point == bench.qp_flops(nodes)
