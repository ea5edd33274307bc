"""The C++ facade (include/cudamonsel_b200.hpp) compiles and links without a GPU.

A LinesOnLayers-style driver (tests/facade/lines_driver.cpp) and a program touching the rest of the
reference's API the facade keeps (tests/facade/api_surface.cpp) are compiled with g++ against the header
and linked against the in-tree libcudamonsel_b200.so; run here, without a GPU, a program fails loudly
with the engine's error (no CPU fallback).
"""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "cudamonsel_b200")


def compile_driver(src, out):
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), src, "-L", LIBDIR,
           "-lcudamonsel_b200", "-Wl,-rpath," + LIBDIR, "-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    return out


@pytest.fixture(scope="module")
def built(tmp_path_factory):
    if not os.path.exists(os.path.join(LIBDIR, "libcudamonsel_b200.so")):
        pytest.skip("library not built")
    d = tmp_path_factory.mktemp("facade")
    return {name: compile_driver(os.path.join(ROOT, "tests", "facade", name + ".cpp"), str(d / name))
            for name in ("lines_driver", "api_surface")}


def test_drivers_compile_and_link(built):
    for exe in built.values():
        assert os.access(exe, os.X_OK)


def test_without_a_gpu_the_driver_fails_loudly(built):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    r = subprocess.run([built["lines_driver"], "x", "1", "1", "1"], capture_output=True, text=True)
    assert r.returncode != 0
    assert "cm_context_create" in r.stderr
