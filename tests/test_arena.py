"""The serving loop's HBM arena (lenstool-hpc_b200/csrc/lt_arena.h), checked on the CPU
by a compiled driver against a byte-map model."""
import pathlib
import subprocess

import pytest

ROOT = pathlib.Path(__file__).resolve().parent.parent


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_arena_model(tmp_path, seed):
    exe = tmp_path / "arena_driver"
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-I", str(ROOT / "lenstool-hpc_b200" / "csrc"),
                    str(ROOT / "tests" / "arena_driver.cpp"), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe), str(seed)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr
