"""The reference's JNI glue (src/jni/dr_inference_hawkes_NativeHPHSingleton.cpp,
the entry points BEAST binds), compiled unmodified against a stub <jni.h>
into oracle/_ref/libhphjni.so together with the reference's hph::factory
(src/factory.cpp) and this engine's factory shim, driven here through ctypes
in place of a JVM.

initialize with the OPENCL flag reaches the CUDA engine through the factory's
GPU slot; without it, the reference's own CPU engine.  Both get the same
events (through jni_harness_set_data, the setters the glue leaves commented
out) and parameters (through the glue's setParameters), and the glue's
getSumOfIncrements must agree: 1e-10 relative in double precision, and the
FLOAT flag (the CUDA engine's plain FP32 mode against the reference's float
engine) within the float-mode bar of 5e-6.
"""
import ctypes
import os

import numpy as np
import pytest

import oracle
from hawkes_b200 import workloads

pytestmark = pytest.mark.gpu

JNI_LIB = os.path.join(os.path.dirname(oracle.REF_LIB), "libhphjni.so")
OPENCL, FLOAT = 1 << 4, 1 << 2
_dp = ctypes.POINTER(ctypes.c_double)


class DoubleArray(ctypes.Structure):
    """The stub's jdoubleArray: {length, data}."""
    _fields_ = [("length", ctypes.c_int32), ("data", _dp)]


@pytest.fixture(scope="module")
def jni():
    if not os.path.exists(JNI_LIB):
        pytest.skip("oracle/_ref/libhphjni.so not built (needs the reference sources)")
    return load_jni()


def load_jni():
    """The glue's entry points and the harness's data setter, with ctypes
    signatures, and a stub JNIEnv pointer."""
    lib = ctypes.CDLL(JNI_LIB)
    p = "Java_dr_inference_hawkes_NativeHPHSingleton_"
    env, obj = ctypes.c_void_p, ctypes.c_void_p
    sig = {
        "initialize": (ctypes.c_int32, [env, obj, ctypes.c_int32, ctypes.c_int32, ctypes.c_int64,
                                        ctypes.c_int32, ctypes.c_int32]),
        "setParameters": (None, [env, obj, ctypes.c_int32, ctypes.POINTER(DoubleArray)]),
        "getSumOfIncrements": (ctypes.c_double, [env, obj, ctypes.c_int32]),
        "getInternalDimension": (ctypes.c_int32, [env, obj, ctypes.c_int32]),
        "storeState": (None, [env, obj, ctypes.c_int32]),
        "acceptState": (None, [env, obj, ctypes.c_int32]),
    }
    fns = {}
    for name, (res, args) in sig.items():
        f = getattr(lib, p + name)
        f.restype, f.argtypes = res, args
        fns[name] = f
    lib.jni_harness_set_data.restype = ctypes.c_int
    lib.jni_harness_set_data.argtypes = [ctypes.c_int, _dp, ctypes.c_size_t, _dp, ctypes.c_size_t]
    fns["set_data"] = lib.jni_harness_set_data
    env_buf = ctypes.create_string_buffer(16)  # the stub JNIEnv holds no state
    fns["env"] = ctypes.cast(env_buf, ctypes.c_void_p)
    fns["_keep"] = (lib, env_buf)
    return fns


def instance(jni, flags, loc, t, p):
    env = jni["env"]
    k = jni["initialize"](env, None, loc.shape[1], loc.shape[0], flags, 0, 0)
    locf = np.ascontiguousarray(loc, dtype=np.float64).reshape(-1)
    tf = np.ascontiguousarray(t, dtype=np.float64)
    assert jni["set_data"](k, locf.ctypes.data_as(_dp), locf.size, tf.ctypes.data_as(_dp),
                           tf.size) == 0
    params = np.ascontiguousarray(p, dtype=np.float64)
    arr = DoubleArray(params.size, params.ctypes.data_as(_dp))
    jni["setParameters"](env, None, k, ctypes.byref(arr))
    return k


def test_jni_glue_reaches_the_cuda_engine(jni):
    loc, t = workloads.uniform(2000, seed=31)
    p = workloads.BASE_PARAMS * np.array([1.1, 0.9, 1.2, 0.8, 1.0, 1.3])
    env = jni["env"]
    cpu = instance(jni, 0, loc, t, p)
    gpu = instance(jni, OPENCL, loc, t, p)
    ll_cpu = jni["getSumOfIncrements"](env, None, cpu)
    ll_gpu = jni["getSumOfIncrements"](env, None, gpu)
    print(f"\nJNI getSumOfIncrements: CPU engine {ll_cpu!r}, CUDA engine {ll_gpu!r}")
    assert abs(ll_gpu - ll_cpu) <= 1e-10 * abs(ll_cpu)
    assert jni["getInternalDimension"](env, None, gpu) == 2
    jni["storeState"](env, None, gpu)
    jni["acceptState"](env, None, gpu)
    assert jni["getSumOfIncrements"](env, None, gpu) == ll_gpu


def test_jni_glue_float_flag(jni):
    loc, t = workloads.uniform(1500, seed=32)
    p = workloads.BASE_PARAMS
    env = jni["env"]
    cpu = instance(jni, FLOAT, loc, t, p)
    gpu = instance(jni, OPENCL | FLOAT, loc, t, p)
    ll_cpu = jni["getSumOfIncrements"](env, None, cpu)
    ll_gpu = jni["getSumOfIncrements"](env, None, gpu)
    print(f"\nJNI FLOAT: CPU float engine {ll_cpu!r}, CUDA plain FP32 {ll_gpu!r}")
    assert abs(ll_gpu - ll_cpu) <= 5e-6 * abs(ll_cpu)
