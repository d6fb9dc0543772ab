"""The header-only C++ drop-in (include/mdx/mdiscr.cuh): a program written
against the reference's template signatures, with its own functors (a mask,
remainders, a non-remainder class function, 8-byte records, arrays of LEN
values, 16-byte records, a three-array tuple whose class reads every field), runs the plain,
segmented, array and tuple templates and checks them against a CPU stable
partition.  Its first case injects a failure of the template's workspace
allocation (host side, no GPU fault) and expects the call to report it and
the next call to succeed."""
import subprocess

import pytest

pytestmark = pytest.mark.gpu


def test_template_dropin_program(cuda_ready):
    from mdiscriminator_b200 import build as mdx_build
    exe = mdx_build.build_cpp_test()
    res = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    print(res.stdout)
    assert res.returncode == 0, res.stdout + res.stderr
    assert "INVALID" not in res.stdout
    assert res.stdout.count("VALID") == 13
    assert "workspace allocation failure: REPORTED" in res.stdout
