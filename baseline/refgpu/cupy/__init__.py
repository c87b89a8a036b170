"""Minimal stand-in for the part of CuPy that the reference's GPU path uses.

BASELINE INFRASTRUCTURE ONLY: it lets the unmodified reference package
(installed under ``baseline/_ref``) run its own GPU code on this machine, where
CuPy is not installed, so that its solve can be timed beside this package's.
Nothing in ``symplectic-stiefel-nearness_b200`` imports it.

The reference compiles its ``.cu`` sources with ``cupy.RawModule(code=...,
options=("--std=c++17",), backend="nvrtc")`` and launches the kernels with
``kernel(grid, block, args)`` on the default stream, where ``args`` are
``numpy.uint64`` device pointers and ``numpy.int32`` / ``numpy.int64``
scalars (src/symplectic_projection/cuda_kernels.py:6-20).  This module
provides exactly that over NVRTC and the CUDA driver API from cuda-python:
the source is compiled to a cubin for the current device, loaded into the
current (PyTorch primary) context, and each launch goes to the legacy default
stream, which PyTorch's default stream also is.  ``__version__`` and
``cuda.runtime.runtimeGetVersion`` cover the reference's environment report.
"""
from __future__ import annotations

import ctypes

import numpy as np
from cuda.bindings import driver, nvrtc

__version__ = "0+nvrtc-stand-in"


def _check(result, what):
    err = result[0] if isinstance(result, tuple) else result
    if int(err) != 0:
        raise RuntimeError(f"{what} failed: {err}")
    return result[1:] if isinstance(result, tuple) and len(result) > 1 else None


def _device_arch():
    _check(driver.cuInit(0), "cuInit")
    (dev,) = _check(driver.cuCtxGetDevice(), "cuCtxGetDevice")
    (major,) = _check(driver.cuDeviceGetAttribute(
        driver.CUdevice_attribute.CU_DEVICE_ATTRIBUTE_COMPUTE_CAPABILITY_MAJOR, dev), "attribute")
    (minor,) = _check(driver.cuDeviceGetAttribute(
        driver.CUdevice_attribute.CU_DEVICE_ATTRIBUTE_COMPUTE_CAPABILITY_MINOR, dev), "attribute")
    return f"sm_{major}{minor}"


class RawModule:
    """cupy.RawModule(code=..., options=..., backend="nvrtc"): NVRTC to a cubin, then cuModuleLoadData."""

    def __init__(self, code, options=(), backend="nvrtc", **_):
        if backend != "nvrtc":
            raise ValueError("only the nvrtc backend is provided")
        (prog,) = _check(nvrtc.nvrtcCreateProgram(code.encode(), b"module.cu", 0, [], []), "nvrtcCreateProgram")
        opts = [o.encode() for o in options] + [f"--gpu-architecture={_device_arch()}".encode()]
        err = nvrtc.nvrtcCompileProgram(prog, len(opts), opts)
        if int(err[0]) != 0:
            (size,) = _check(nvrtc.nvrtcGetProgramLogSize(prog), "log size")
            log = b" " * size
            nvrtc.nvrtcGetProgramLog(prog, log)
            raise RuntimeError(f"NVRTC compilation failed:\n{log.decode(errors='replace')}")
        (size,) = _check(nvrtc.nvrtcGetCUBINSize(prog), "nvrtcGetCUBINSize")
        image = b" " * size
        _check(nvrtc.nvrtcGetCUBIN(prog, image), "nvrtcGetCUBIN")
        nvrtc.nvrtcDestroyProgram(prog)
        (self._module,) = _check(driver.cuModuleLoadData(image), "cuModuleLoadData")

    def get_function(self, name):
        (fn,) = _check(driver.cuModuleGetFunction(self._module, name.encode()), f"cuModuleGetFunction({name})")
        return RawKernel(fn)


class RawKernel:
    """kernel(grid, block, args): one cuLaunchKernel on the legacy default stream."""

    _CTYPES = {np.uint64: ctypes.c_uint64, np.int64: ctypes.c_int64, np.int32: ctypes.c_int32,
               np.uint32: ctypes.c_uint32, np.float64: ctypes.c_double, np.float32: ctypes.c_float}

    def __init__(self, fn):
        self._fn = fn

    def __call__(self, grid, block, args, shared_mem=0):
        values = []
        for a in args:
            ct = self._CTYPES.get(type(a))
            if ct is None:
                raise TypeError(f"kernel argument of type {type(a).__name__} is not a numpy scalar")
            values.append(ct(a.item()))
        params = (ctypes.c_void_p * max(1, len(values)))(*[ctypes.addressof(v) for v in values])
        g = tuple(grid) + (1,) * (3 - len(grid))
        b = tuple(block) + (1,) * (3 - len(block))
        _check(driver.cuLaunchKernel(self._fn, *g, *b, shared_mem, 0, ctypes.addressof(params), 0),
               "cuLaunchKernel")


class _Runtime:
    @staticmethod
    def runtimeGetVersion():
        (v,) = _check(driver.cuDriverGetVersion(), "cuDriverGetVersion")
        return v


class cuda:  # noqa: N801 - mirrors cupy.cuda
    runtime = _Runtime
