"""Build recipe for libmdx.so (sm_100a) -- run by ``__graft_entry__.build()``.

Compiles ``csrc/mdx_capi.cu`` (which includes every kernel header) with nvcc
directly into ``mdiscriminator_b200/libmdx.so``, in-tree, so the library
travels with the repository snapshot.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libmdx.so")
SOURCES = [os.path.join(HERE, "csrc", "mdx_capi.cu"), os.path.join(HERE, "csrc", "mdx_noalloc.cu"),
           os.path.join(HERE, "csrc", "mdx_server.cu"), os.path.join(HERE, "csrc", "mdx_wide.cu")]
HEADERS_DIRS = [os.path.join(HERE, "csrc"), os.path.join(os.path.dirname(HERE), "include")]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise FileNotFoundError("nvcc not found")
    return cand


def _newest_input_mtime() -> float:
    t = 0.0
    for p in SOURCES:
        t = max(t, os.path.getmtime(p))
    for d in HEADERS_DIRS:
        for root, _, files in os.walk(d):
            for f in files:
                if f.endswith((".cu", ".cuh", ".h")):
                    t = max(t, os.path.getmtime(os.path.join(root, f)))
    t = max(t, os.path.getmtime(__file__))
    return t


def up_to_date() -> bool:
    return os.path.exists(LIB) and os.path.getmtime(LIB) >= _newest_input_mtime()


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return LIB
    cmd = [nvcc(), *ARCH, "-lineinfo", "-O3", "-std=c++17", "-shared", "-Xcompiler", "-fPIC",
           "-Xptxas", "-v" if verbose else "-O3", "-o", LIB + ".tmp", *SOURCES]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + " ".join(cmd) + "\n" + res.stdout + res.stderr)
    if verbose:
        sys.stderr.write(res.stderr)
    os.replace(LIB + ".tmp", LIB)
    return LIB


CPP_TEST_SRC = os.path.join(os.path.dirname(HERE), "tests", "cpp", "template_dropin.cu")
CPP_TEST_BIN = os.path.join(os.path.dirname(HERE), "tests", "cpp", "template_dropin")


def build_cpp_test(force: bool = False) -> str:
    """Compile the program that uses the header-only templates (include/mdx/mdiscr.cuh)."""
    inputs = [CPP_TEST_SRC, os.path.join(os.path.dirname(HERE), "include", "mdx", "mdiscr.cuh")]
    newest = max([os.path.getmtime(p) for p in inputs] + [_newest_input_mtime()])
    if not force and os.path.exists(CPP_TEST_BIN) and os.path.getmtime(CPP_TEST_BIN) >= newest:
        return CPP_TEST_BIN
    cmd = [nvcc(), *ARCH, "-O2", "-std=c++17", "-I", os.path.join(os.path.dirname(HERE), "include"),
           "-o", CPP_TEST_BIN + ".tmp", CPP_TEST_SRC]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + " ".join(cmd) + "\n" + res.stdout + res.stderr)
    os.replace(CPP_TEST_BIN + ".tmp", CPP_TEST_BIN)
    return CPP_TEST_BIN


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
