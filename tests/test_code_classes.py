"""Host check (no GPU) of the haplotype code words behind the packed FP32 kernels' prior tables:
tests/native/code_classes_check.cpp, compiled against the kernels' own header, compares for every
haplotype byte and read byte in both variants the FP64 path's masked compare and the FP32 path's
class-table choice (with the byte compare of class-4 columns for inter rows outside A/C/G/T) with
the match-code compare of the reference semantics."""
from __future__ import annotations

import shutil
import subprocess
from pathlib import Path

import pytest

SRC = Path(__file__).resolve().parent / "native" / "code_classes_check.cpp"


def test_code_words_and_prior_classes_match_byte_semantics(tmp_path):
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("g++ not available")
    exe = tmp_path / "code_classes_check"
    subprocess.run([cxx, "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror", str(SRC), "-o", str(exe)], check=True)
    res = subprocess.run([str(exe)], capture_output=True, text=True)
    assert res.returncode == 0, res.stdout + res.stderr
    assert "0 mismatches" in res.stdout
