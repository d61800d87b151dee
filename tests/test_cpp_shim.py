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
CFD_SRC = os.path.join(ROOT, "tests", "cpp", "test_cfd_interface.cpp")
TURBINE_SRC = os.path.join(ROOT, "tests", "cpp", "test_turbine_interface.cpp")


def _compile(src: str = SRC, name: str = "test_shim", with_oracle: bool = False) -> str:
    """g++ build of a driver against the shim (and, for the cross-checking
    drivers, the oracle library: test infrastructure)."""
    kbuild.build()
    os.makedirs(OUT_DIR, exist_ok=True)
    exe = os.path.join(OUT_DIR, name)
    gxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    cmd = [gxx, "-std=c++20", "-O1", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), src,
           "-L", LIB_DIR, "-lkynema_b200", "-Wl,-rpath," + LIB_DIR, "-o", exe]
    if with_oracle:
        from oracle import oracle_py
        odir = os.path.dirname(oracle_py.build())
        cmd[-2:-2] = ["-I", os.path.join(ROOT, "oracle"), "-L", odir, "-lkyn_oracle", "-Wl,-rpath," + odir]
    subprocess.run(cmd, check=True)
    return exe


def test_shim_compiles():
    assert os.path.exists(_compile())
    assert os.path.exists(_compile(BLADE_SRC, "test_blade_interface"))
    assert os.path.exists(_compile(CFD_SRC, "test_cfd_interface"))
    assert os.path.exists(_compile(TURBINE_SRC, "test_turbine_interface", with_oracle=True))


def test_interface_geometry_helpers():
    """The blade interface's host geometry (no GPU): GLL points, trapezoidal
    quadrature, the end-point-constrained least-squares fit of the reference
    axis and the tangent/twist frame, against independent computations."""
    import numpy as np
    from openturbine_b200.model import CreateTrapezoidalQuadrature, GenerateGLLPoints
    exe = _compile(os.path.join(ROOT, "tests", "cpp", "test_interface_math.cpp"), "test_interface_math")
    out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split("\n")
    vals = {}
    for line in out:
        if line:
            k, *v = line.split()
            vals.setdefault(k, []).append([float(x) for x in v])
    for order in (1, 4, 10):
        got = [v[1] for v in vals["gll"] if int(v[0]) == order]
        np.testing.assert_allclose(got, GenerateGLLPoints(order), rtol=0, atol=1e-14)
    np.testing.assert_allclose(vals["trap"], CreateTrapezoidalQuadrature([0., 0.1, 0.25, 0.6, 1.]),
                               rtol=0, atol=1e-15)
    # the fit: interior rows are the normal equations of the key points, the
    # end rows pin the first and last key point
    xi = np.array(GenerateGLLPoints(4))
    s = np.arange(7) / 6.
    kp = np.stack([10 * s, 0.5 * s * s, 0.1 * s ** 3], axis=1)
    phi = np.array([[np.prod([(2 * si - 1 - xi[m]) / (xi[j] - xi[m]) for m in range(5) if m != j])
                     for si in s] for j in range(5)])
    A = phi @ phi.T
    B = phi @ kp
    A[0] = 0; A[0, 0] = 1; B[0] = kp[0]
    A[-1] = 0; A[-1, -1] = 1; B[-1] = kp[-1]
    np.testing.assert_allclose(vals["fit"], np.linalg.solve(A, B), rtol=0, atol=1e-12)
    # the frame: first axis along the tangent, turned by 30 degrees about it
    w, x, y, z = vals["ttq"][0]
    R = np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
                  [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
                  [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)]])
    t = np.array([1., 2., .5]) / np.linalg.norm([1., 2., .5])
    np.testing.assert_allclose(R[:, 0], t, atol=1e-14)
    e2 = np.array([0., 1., 0.]) - t * t[1]
    e2 /= np.linalg.norm(e2)
    ang = np.radians(30.)
    np.testing.assert_allclose(R[:, 1], np.cos(ang) * e2 + np.sin(ang) * np.cross(t, e2), atol=1e-14)


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


@pytest.mark.gpu
def test_cfd_interface_floating_platform(tmp_path):
    """CFD interface (include/kynema_b200_interfaces.hpp, namespace cfd) on the
    reference's CFDInterfaceTest.PrecessionTest (with SaveState/RestoreState),
    FloatingPlatform (three mooring lines) and Restart, at the tests' 1e-12."""
    exe = _compile(CFD_SRC, "test_cfd_interface")
    r = subprocess.run([exe, str(tmp_path / "restart.dat")], capture_output=True, text=True, timeout=300)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "OK (0 failures)" in r.stdout



def test_turbine_model_description_without_a_gpu():
    """The IEA-15 turbine's model, built by the turbine component on the host
    and described by kyn_model_describe (no device): 371 unknowns condensed to
    a bordered system of 137, DOF counts and CRS graph equal to the oracle's."""
    exe = _compile(TURBINE_SRC, "test_turbine_interface", with_oracle=True)
    golden = os.path.join(ROOT, "tests", "golden")
    r = subprocess.run([exe, os.path.join(golden, "iea15_blade_windio.txt"),
                        os.path.join(golden, "iea15_turbine_windio.txt"), "--describe"],
                       capture_output=True, text=True, timeout=300)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip().endswith("OK")


@pytest.mark.gpu
def test_turbine_interface_iea15_structure():
    """TurbineInterface (include/kynema_b200_interfaces.hpp) on the reference's
    TurbineInterfaceTest.IEA15_Structure: the IEA-15-240-RWT tower, drive train,
    hub and three blades (a condensed dense model), 9 steps under a tower-top
    load, generator torque, pitch and yaw ramps, tower top position at the
    test's 1e-10, and the oracle stepping the same model beside it."""
    exe = _compile(TURBINE_SRC, "test_turbine_interface", with_oracle=True)
    golden = os.path.join(ROOT, "tests", "golden")
    r = subprocess.run([exe, os.path.join(golden, "iea15_blade_windio.txt"),
                        os.path.join(golden, "iea15_turbine_windio.txt")],
                       capture_output=True, text=True, timeout=600)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip().endswith("OK")
