"""Shared helpers for the tests: device transfers and tolerances."""
import numpy as np

# Tolerances. FP64 results: rel-L2 1e-12 against the FP64 oracle and the
# reference tests' 1e-10 max-abs on their shapes (test/c2c/test_fftw_c2c_nd.cpp:119).
# FP32 results: rel-L2 2e-6 against the FP64 oracle, and the reference float
# tests' 1e-4 * peak|ref| max-abs rule (test/c2c/test_fftw_c2c_nd_float.cpp:101-106).
REL_F64 = 1e-12
REL_F32 = 2e-6
ABS_F64 = 1e-10


def tol(prec) -> float:
    return REL_F64 if prec == 1 else REL_F32


def to_dev(a: np.ndarray):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def to_host(t) -> np.ndarray:
    import torch
    torch.cuda.synchronize()
    return t.cpu().numpy()


def cdtype(prec):
    return np.complex128 if prec == 1 else np.complex64


def rdtype(prec):
    return np.float64 if prec == 1 else np.float32
