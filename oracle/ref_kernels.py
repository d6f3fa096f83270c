"""The reference's own CUDA pair kernel, run as a checker -- TEST INFRASTRUCTURE ONLY.

``oracle/Makefile`` (target ``ref``) compiles the reference's chart-driven pair-integration
kernels (crates/sonium-compute/src/cuda/kernels/bem_kernels.cu) unchanged into
``oracle/_ref/bem_kernels.cubin``. This module loads that module through the CUDA runtime's
library API and launches ``sonium_bem_quadrature_pair_c64`` exactly as the reference's backend
does (crates/sonium-compute/src/cuda/cublas.rs:4640-4720: 128 threads per block, one thread per
pair, pair/output offset 0 and stride 1), on charts built by the oracle (``oracle.chart``, the
restatement of tbem.rs:4998-5161). Only the tests and the reference-GPU baseline leg of
``bench.py`` use it; the product library never does.
"""
from __future__ import annotations

import ctypes as ct
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
CUBIN = os.path.join(_HERE, "_ref", "bem_kernels.cubin")
KERNEL = b"sonium_bem_quadrature_pair_c64"
BLOCK = 128  # the reference backend's block size for this kernel (cublas.rs:4692)


def build() -> str | None:
    """Compile the reference kernels when the reference tree is present (idempotent); returns the
    cubin path, or None when neither the tree nor a prebuilt cubin is there."""
    src = os.path.join(os.environ.get("REF_ROOT", "/root/reference"),
                       "crates/sonium-compute/src/cuda/kernels/bem_kernels.cu")
    if os.path.exists(src):
        subprocess.run(["make", "-s", "-C", _HERE, "ref"], check=True)
    return CUBIN if os.path.exists(CUBIN) else None


class _Dim3(ct.Structure):
    _fields_ = [("x", ct.c_uint), ("y", ct.c_uint), ("z", ct.c_uint)]


def _cudart():
    for name in ("libcudart.so.12", "libcudart.so", "/usr/local/cuda/lib64/libcudart.so.12"):
        try:
            rt = ct.CDLL(name)
            break
        except OSError:
            continue
    else:
        raise RuntimeError("libcudart not found")
    P = ct.c_void_p
    rt.cudaSetDevice.argtypes = [ct.c_int]
    rt.cudaMalloc.argtypes = [ct.POINTER(P), ct.c_size_t]
    rt.cudaFree.argtypes = [P]
    rt.cudaMemcpy.argtypes = [P, P, ct.c_size_t, ct.c_int]
    rt.cudaLibraryLoadFromFile.argtypes = [ct.POINTER(P), ct.c_char_p, P, P, ct.c_uint, P, P, ct.c_uint]
    rt.cudaLibraryGetKernel.argtypes = [ct.POINTER(P), P, ct.c_char_p]
    rt.cudaLaunchKernel.argtypes = [P, _Dim3, _Dim3, ct.POINTER(P), ct.c_size_t, P]
    rt.cudaEventCreate.argtypes = [ct.POINTER(P)]
    rt.cudaEventRecord.argtypes = [P, P]
    rt.cudaEventSynchronize.argtypes = [P]
    rt.cudaEventElapsedTime.argtypes = [ct.POINTER(ct.c_float), P, P]
    rt.cudaEventDestroy.argtypes = [P]
    rt.cudaGetErrorString.argtypes = [ct.c_int]
    rt.cudaGetErrorString.restype = ct.c_char_p
    return rt


class RefPairKernel:
    """sonium_bem_quadrature_pair_c64 from the reference's source, loaded on one device."""

    def __init__(self, device: int = 0):
        if not os.path.exists(CUBIN):
            raise RuntimeError(f"{CUBIN} is missing: build it with `make -C oracle ref` where the reference "
                               "tree is present")
        self.rt = _cudart()
        self._ok(self.rt.cudaSetDevice(device), "cudaSetDevice")
        self.lib = ct.c_void_p()
        self._ok(self.rt.cudaLibraryLoadFromFile(ct.byref(self.lib), CUBIN.encode(), None, None, 0, None, None, 0),
                 "cudaLibraryLoadFromFile")
        self.kernel = ct.c_void_p()
        self._ok(self.rt.cudaLibraryGetKernel(ct.byref(self.kernel), self.lib, KERNEL), "cudaLibraryGetKernel")

    def _ok(self, rc, what):
        if rc != 0:
            raise RuntimeError(f"{what} failed: {self.rt.cudaGetErrorString(rc).decode()}")

    def _alloc(self, nbytes):
        p = ct.c_void_p()
        self._ok(self.rt.cudaMalloc(ct.byref(p), max(int(nbytes), 16)), "cudaMalloc")
        return p

    def run(self, pairs: np.ndarray, samples: np.ndarray, k: float, harmonic_factor: float = 1.0,
            reps: int = 1):
        """Channels (G, H, H^T, E) of every pair, (n_pairs, 4) complex128, and the average kernel
        time in ms over `reps` launches (CUDA events around the launches on the default stream)."""
        n = int(pairs.shape[0])
        if n == 0:
            return np.zeros((0, 4), np.complex128), 0.0
        pairs = np.ascontiguousarray(pairs)
        # the reference uploads one default sample when a chart holds none (cublas.rs:4659-4663)
        samples = np.ascontiguousarray(samples) if samples.shape[0] else np.zeros(1, samples.dtype)
        rt = self.rt
        d_pairs, d_samples, d_out = self._alloc(pairs.nbytes), self._alloc(samples.nbytes), self._alloc(64 * n)
        e0, e1 = ct.c_void_p(), ct.c_void_p()
        try:
            self._ok(rt.cudaMemcpy(d_pairs, pairs.ctypes.data, pairs.nbytes, 1), "cudaMemcpy")
            self._ok(rt.cudaMemcpy(d_samples, samples.ctypes.data, samples.nbytes, 1), "cudaMemcpy")
            a_k, a_h = ct.c_double(k), ct.c_double(harmonic_factor)
            a_ns, a_np = ct.c_uint64(samples.shape[0]), ct.c_uint64(n)
            zero, one = ct.c_uint64(0), ct.c_uint64(1)
            args = (ct.c_void_p * 11)(*[ct.cast(ct.byref(v), ct.c_void_p) for v in (
                d_pairs, d_samples, d_out, a_k, a_h, a_ns, a_np, zero, one, zero, one)])
            grid, block = _Dim3((n + BLOCK - 1) // BLOCK, 1, 1), _Dim3(BLOCK, 1, 1)
            self._ok(rt.cudaEventCreate(ct.byref(e0)), "cudaEventCreate")
            self._ok(rt.cudaEventCreate(ct.byref(e1)), "cudaEventCreate")
            self._ok(rt.cudaEventRecord(e0, None), "cudaEventRecord")
            for _ in range(max(1, reps)):
                self._ok(rt.cudaLaunchKernel(self.kernel, grid, block, args, 0, None), "cudaLaunchKernel")
            self._ok(rt.cudaEventRecord(e1, None), "cudaEventRecord")
            self._ok(rt.cudaEventSynchronize(e1), "cudaEventSynchronize")
            ms = ct.c_float()
            self._ok(rt.cudaEventElapsedTime(ct.byref(ms), e0, e1), "cudaEventElapsedTime")
            out = np.zeros((n, 4), np.complex128)
            self._ok(rt.cudaMemcpy(out.ctypes.data, d_out, out.nbytes, 2), "cudaMemcpy")
            return out, ms.value / max(1, reps)
        finally:
            for e in (e0, e1):
                if e:
                    rt.cudaEventDestroy(e)
            for p in (d_pairs, d_samples, d_out):
                rt.cudaFree(p)
