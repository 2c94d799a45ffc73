"""CPU side of the reference's JNI glue build (oracle/_ref/libhphjni.so, see
test_jni_gpu.py): the library loads without a GPU, exports the entry points
the glue defines, and its CPU engine path (initialize without the OPENCL
flag) gives the oracle's log-likelihood."""
import ctypes
import os

import numpy as np
import pytest

import oracle
from hawkes_b200 import workloads

JNI_LIB = os.path.join(os.path.dirname(oracle.REF_LIB), "libhphjni.so")
ENTRY_POINTS = ("initialize", "getSumOfIncrements", "storeState", "restoreState",
                "acceptState", "setParameters", "getInternalDimension")

pytestmark = pytest.mark.skipif(not os.path.exists(JNI_LIB),
                                reason="oracle/_ref/libhphjni.so not built")


def test_jni_exports():
    lib = ctypes.CDLL(JNI_LIB)
    for name in ENTRY_POINTS:
        assert hasattr(lib, "Java_dr_inference_hawkes_NativeHPHSingleton_" + name), name


def test_jni_cpu_engine_matches_oracle():
    import test_jni_gpu as g
    jni = g.load_jni()
    loc, t = workloads.uniform(800, seed=33)
    p = workloads.BASE_PARAMS
    k = g.instance(jni, 0, loc, t, p)
    ll = jni["getSumOfIncrements"](jni["env"], None, k)
    o = oracle.oracle_eval(loc, t, p, threads=2)
    assert abs(ll - o["loglik"]) <= 1e-12 * abs(o["loglik"])
