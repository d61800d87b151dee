"""The reference's regression drivers written against the C++ host shim
(include/kynema_b200.hpp) and its blade interface
(include/kynema_b200_interfaces.hpp), compiled with g++ and run on the GPU.

The CPU test only compiles the driver, so a broken header fails without a GPU.
"""
import os
import subprocess

import pytest

from openturbine_b200 import build as kbuild

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "test_shim.cpp")
OUT_DIR = os.path.join(ROOT, "tests", "cpp", "_build")
LIB_DIR = os.path.join(ROOT, "openturbine_b200", "_lib")


BLADE_SRC = os.path.join(ROOT, "tests", "cpp", "test_blade_interface.cpp")


def _compile(src: str = SRC, name: str = "test_shim") -> str:
    kbuild.build()
    os.makedirs(OUT_DIR, exist_ok=True)
    exe = os.path.join(OUT_DIR, name)
    gxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    cmd = [gxx, "-std=c++20", "-O1", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), src,
           "-L", LIB_DIR, "-lkynema_b200", "-Wl,-rpath," + LIB_DIR, "-o", exe]
    subprocess.run(cmd, check=True)
    return exe


def test_shim_compiles():
    assert os.path.exists(_compile())
    assert os.path.exists(_compile(BLADE_SRC, "test_blade_interface"))


@pytest.mark.gpu
def test_blade_interface_rotating_beam_and_windio():
    """BladeInterface (include/kynema_b200_interfaces.hpp) on the reference's
    BladeInterfaceTest.RotatingBeam (root and tip motion) and BladeWindIO (the
    IEA-15 blade from its WindIO description, tip position), both at 1e-10."""
    exe = _compile(BLADE_SRC, "test_blade_interface")
    fixture = os.path.join(ROOT, "tests", "golden", "iea15_blade_windio.txt")
    r = subprocess.run([exe, fixture], capture_output=True, text=True, timeout=300)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "OK (0 failures)" in r.stdout


@pytest.mark.gpu
def test_shim_cantilever_and_rotating_beam():
    exe = _compile()
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "OK (0 failures)" in r.stdout
