"""CPU checkers for the stable m-way partition -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg import this package.  The product path (``mdiscriminator_b200``) never
does: it fails loudly when its CUDA library is missing instead of falling back
to anything here.

Two libraries:

* ``libmdx_oracle.so`` -- the C restatement of the reference's ``seqMdiscr``
  (``cuda_code/SeqMdiscr.h:10-57``); see ``mdx_oracle.c`` for the line map.
* ``_ref/libref_mdiscr.so`` -- the reference's own ``SeqMdiscr.h`` and
  ``OpenmpMdiscr.h`` compiled from its sources through ``ref_shim.cpp``.  Used
  to pin the restatement and as the timed CPU baseline.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "libmdx_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libref_mdiscr.so")

DISCR_MOD = 0
DISCR_MASK = 1

_u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")

_lib = None
_ref = None


def reference_sources() -> str | None:
    """The reference checkout's ``cuda_code/`` directory, or None.

    ``MDX_REF_SRC`` names it; otherwise a checkout named ``reference`` beside
    the repository directory is used when it holds ``SeqMdiscr.h``."""
    env = os.environ.get("MDX_REF_SRC")
    if env:
        return env
    beside = os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference", "cuda_code")
    return beside if os.path.exists(os.path.join(beside, "SeqMdiscr.h")) else None


def build(quiet: bool = True) -> None:
    """Compile the oracle (and, where the reference sources exist, _ref)."""
    cmd = ["make", "-C", HERE]
    src = reference_sources()
    if src:
        cmd.append(f"REF_SRC={src}")
    out = subprocess.run(cmd, capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)
    if not quiet:
        print(out.stdout)


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            build()
        L = ctypes.CDLL(ORACLE_SO)
        vp = ctypes.c_void_p
        L.mdx_oracle_partition_u32.argtypes = [ctypes.c_uint64, _u32p, _u32p, ctypes.c_int,
                                               ctypes.c_uint32, vp, vp]
        L.mdx_oracle_partition_u32.restype = ctypes.c_int
        L.mdx_oracle_partition_rec8.argtypes = [ctypes.c_uint64, _u64p, _u64p, ctypes.c_int,
                                                ctypes.c_uint32, vp, vp]
        L.mdx_oracle_partition_rec8.restype = ctypes.c_int
        L.mdx_oracle_partition_segmented.argtypes = [ctypes.c_uint64, vp, vp, ctypes.c_size_t,
                                                     _u64p, ctypes.c_uint64, ctypes.c_int,
                                                     ctypes.c_uint32, vp, vp]
        L.mdx_oracle_partition_segmented.restype = ctypes.c_int
        L.mdx_oracle_flags_to_offsets.argtypes = [ctypes.c_uint64, _i32p, _u64p, ctypes.c_uint64]
        L.mdx_oracle_flags_to_offsets.restype = ctypes.c_int64
        L.mdx_oracle_tuple_to_headflags.argtypes = [ctypes.c_uint64, _u32p, ctypes.c_uint32, _u32p]
        L.mdx_oracle_tuple_to_headflags.restype = None
        L.mdx_oracle_fill_uniform_u32.argtypes = [ctypes.c_uint64, ctypes.c_uint64, _u32p]
        L.mdx_oracle_fill_uniform_u32.restype = None
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def partition(values: np.ndarray, m: int, kind: int = DISCR_MOD, headflags: bool = False):
    """Stable partition of a u32 array or a (n,) u64 record array (key = low word).

    Returns ``(out, sizes)`` or ``(out, sizes, flags)``.
    """
    values = np.ascontiguousarray(values)
    n = values.shape[0]
    out = np.empty_like(values)
    sizes = np.zeros(m, dtype=np.uint32)
    flags = np.zeros(n, dtype=np.uint32) if headflags else None
    if values.dtype == np.uint32:
        rc = lib().mdx_oracle_partition_u32(n, values, out, kind, m, _ptr(sizes), _ptr(flags))
    elif values.dtype == np.uint64:
        rc = lib().mdx_oracle_partition_rec8(n, values, out, kind, m, _ptr(sizes), _ptr(flags))
    else:
        raise TypeError(f"unsupported dtype {values.dtype}")
    if rc != 0:
        raise ValueError("oracle rejected the arguments")
    return (out, sizes, flags) if headflags else (out, sizes)


def partition_segmented(values: np.ndarray, offsets: np.ndarray, m: int,
                        kind: int = DISCR_MOD, headflags: bool = False):
    """Per-segment stable partition; returns ``(out, seg_sizes[S, m][, flags])``."""
    values = np.ascontiguousarray(values)
    offsets = np.ascontiguousarray(offsets, dtype=np.uint64)
    n = values.shape[0]
    S = offsets.shape[0] - 1
    out = np.empty_like(values)
    seg_sizes = np.zeros((S, m), dtype=np.uint32)
    flags = np.zeros(n, dtype=np.uint32) if headflags else None
    rc = lib().mdx_oracle_partition_segmented(n, _ptr(values), _ptr(out), values.itemsize,
                                              offsets, S, kind, m, _ptr(seg_sizes), _ptr(flags))
    if rc != 0:
        raise ValueError("oracle rejected the arguments")
    return (out, seg_sizes, flags) if headflags else (out, seg_sizes)


def flags_to_offsets(flags: np.ndarray) -> np.ndarray:
    flags = np.ascontiguousarray(flags, dtype=np.int32)
    n = flags.shape[0]
    offs = np.zeros(n + 1, dtype=np.uint64)
    S = lib().mdx_oracle_flags_to_offsets(n, flags, offs, n)
    if S < 0:
        raise ValueError("malformed head-flag segment sizes")
    return offs[: S + 1].copy()


def tuple_to_headflags(sizes: np.ndarray, n: int) -> np.ndarray:
    sizes = np.ascontiguousarray(sizes, dtype=np.uint32)
    out = np.zeros(n, dtype=np.uint32)
    lib().mdx_oracle_tuple_to_headflags(n, sizes, sizes.shape[0], out)
    return out


def fill_uniform_u32(n: int, seed: int) -> np.ndarray:
    out = np.empty(n, dtype=np.uint32)
    lib().mdx_oracle_fill_uniform_u32(n, seed, out)
    return out


# ---------------------------------------------------------------- reference --
def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref() -> ctypes.CDLL:
    global _ref
    if _ref is None:
        if not ref_available():
            raise FileNotFoundError(REF_SO)
        R = ctypes.CDLL(REF_SO)
        vp = ctypes.c_void_p
        R.ref_seq_mdiscr_u32.argtypes = [ctypes.c_uint, ctypes.c_uint, _u32p, _u32p, _u32p,
                                         ctypes.c_int, ctypes.c_int]
        R.ref_seq_mdiscr_u32.restype = ctypes.c_long
        R.ref_seq_mdiscr_rec8.argtypes = [ctypes.c_uint, ctypes.c_uint, vp, vp, _u32p, ctypes.c_int]
        R.ref_seq_mdiscr_rec8.restype = ctypes.c_long
        R.ref_openmp_mdiscr_u32.argtypes = [ctypes.c_uint, ctypes.c_uint, _u32p, _u32p, _i32p,
                                            ctypes.c_int]
        R.ref_openmp_mdiscr_u32.restype = ctypes.c_long
        R.ref_openmp_max_threads.argtypes = []
        R.ref_openmp_max_threads.restype = ctypes.c_int
        _ref = R
    return _ref


def ref_seq(values: np.ndarray, m: int, specialized: bool = False, measure: bool = False):
    """The reference's seqMdiscr<Mod<m>> (or Mod4/Mod8 when ``specialized``).

    Returns ``(out, headflags[n], runtime_us)``; headflags has the reference's
    form (the one-past-end slot it may write is dropped).
    """
    values = np.ascontiguousarray(values)
    n = values.shape[0]
    out = np.empty_like(values)
    flags = np.zeros(n + 1, dtype=np.uint32)
    if values.dtype == np.uint32:
        rc = ref().ref_seq_mdiscr_u32(m, n, values, out, flags, int(specialized), int(measure))
    else:
        rc = ref().ref_seq_mdiscr_rec8(m, n, _ptr(values), _ptr(out), flags, int(measure))
    if rc == -2:
        raise ValueError(f"reference shim not instantiated for m={m}")
    return out, flags[:n].copy(), rc


def ref_openmp(values: np.ndarray, m: int, threads: int = 0):
    """The reference's openmpMdiscr; returns ``(out, headflags, runtime_us)``."""
    values = np.ascontiguousarray(values, dtype=np.uint32)
    n = values.shape[0]
    out = np.empty_like(values)
    flags = np.zeros(n, dtype=np.int32)
    us = ref().ref_openmp_mdiscr_u32(m, n, values, out, flags, threads)
    if us == -2:
        raise ValueError(f"reference shim not instantiated for m={m}")
    return out, flags, us
