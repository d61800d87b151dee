"""Extract the reference's golden vectors into JSON fixtures.

Run where the reference tree is present, giving its root directory:
    python tests/golden/make_golden.py <reference root>
(or set KYN_REFERENCE_ROOT instead of the argument).
It reads the reference's own test sources as text, pulls the numeric
literals of the named initialisers, and writes tests/golden/*.json.  The GPU
box never reads the reference; tests use only the committed JSON.

Sources (paths relative to the reference project root):
  tests/regression_tests/regression/iea15_rotor_data.hpp   IEA-15 rotor inputs
  tests/regression_tests/regression/test_rotor.cpp:150-189   IEA-15 expected q
  tests/regression_tests/regression/test_cantilever_beam.cpp expected tip q
  tests/regression_tests/regression/test_solver.cpp          assembled b, x, err
  tests/regression_tests/regression/test_rotating_beam.cpp   expected q (prescribed
                                                             root; rotation control;
                                                             revolute joint, generator
                                                             torque)
  tests/unit_tests/system/beams/test_curved_beam.hpp         kernel-level data
  tests/regression_tests/interfaces/test_blade_interface.cpp + its WindIO file
                                                             IEA-15 blade input, tip
  tests/unit_tests/constraints/test_calculate_revolute_joint_*.cpp
                                                             revolute joint kernels
  tests/regression_tests/interfaces/test_cfd_interface.cpp    floating platform q
                                                             (mass, mooring springs)
  tests/regression_tests/regression/test_heavy_top.cpp         heavy top q (three-row
                                                             constraints)
  tests/regression_tests/regression/test_masses.cpp,
    test_precession.cpp, test_spring_mass_system.cpp          point masses, springs
"""
from __future__ import annotations

import json
import os
import re
import sys

NUM = r"[-+]?(?:\d+\.\d*|\.\d+|\d+)(?:[eE][-+]?\d+)?"


def strip_comments(text: str) -> str:
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return re.sub(r"//[^\n]*", "", text)


def _block(text: str, start: int) -> str:
    """Return the balanced {...} block beginning at the first '{' after start."""
    i = text.index("{", start)
    depth = 0
    for j in range(i, len(text)):
        if text[j] == "{":
            depth += 1
        elif text[j] == "}":
            depth -= 1
            if depth == 0:
                return text[i : j + 1]
    raise ValueError("unbalanced braces")


def numbers_of(text: str, name: str, known: dict | None = None) -> list[float]:
    m = re.search(r"\b" + re.escape(name) + r"\b[^=;{]*=", text)
    if not m:
        raise KeyError(name)
    blk = _block(text, m.end())
    # resolve element references to other initialisers, e.g. kStrainInterpolationHolder[2]
    if known:
        def sub(mm):
            return repr(known[mm.group(1)][int(mm.group(2))])
        blk = re.sub(r"\b(\w+)\[(\d+)\]", lambda mm: sub(mm) if mm.group(1) in known
                     else mm.group(0), blk)
        blk = re.sub(r"-\s*-", "", blk)
    # drop template arguments like std::array<double, 3> inside initialisers
    blk = re.sub(r"std::array<[^>]*>", "", blk)
    blk = re.sub(r"std::array\b", "", blk)
    return [float(x) for x in re.findall(NUM, blk)]


def expect_near_values(text: str, start_pat: str, stop_pat: str) -> list[tuple[str, float]]:
    i = text.index(start_pat)
    j = text.index(stop_pat, i)
    out = []
    for m in re.finditer(r"EXPECT_NEAR\(\s*q\((\d+),\s*(\d+)\),\s*(" + NUM + r"|q\(\d+,\s*\d+\))",
                         text[i:j]):
        out.append((m.group(1), m.group(2), m.group(3)))
    return out


def view_after(text: str, anchor: str, occurrence: int = 0) -> list[float]:
    """Numbers of the brace block passed to the expect_* call after `anchor`."""
    pos = -1
    for _ in range(occurrence + 1):
        pos = text.index(anchor, pos + 1)
    return [float(x) for x in re.findall(NUM, _block(text, pos))]


def main(ref: str) -> None:
    out_dir = os.path.dirname(os.path.abspath(__file__))
    reg = os.path.join(ref, "tests", "regression_tests", "regression")
    unit = os.path.join(ref, "tests", "unit_tests", "system", "beams")

    # ---- IEA-15 rotor ----------------------------------------------------
    rd = strip_comments(open(os.path.join(reg, "iea15_rotor_data.hpp")).read())
    node_xi = numbers_of(rd, "node_xi")
    coords = numbers_of(rd, "node_coords")
    quad = numbers_of(rd, "trapz_quadrature")
    secs = numbers_of(rd, "material_sections")
    assert len(coords) == 7 * len(node_xi)
    assert len(secs) % 73 == 0
    sections = []
    for k in range(len(secs) // 73):
        s = secs[73 * k : 73 * (k + 1)]
        sections.append({"position": s[0], "M_star": s[1:37], "C_star": s[37:73]})
    rt = strip_comments(open(os.path.join(reg, "test_rotor.cpp")).read())
    exp = []
    for node, comp, val in expect_near_values(rt, "TEST(RotorTest, IEA15Rotor)",
                                              "TEST(RotorTest, IEA15RotorHub)"):
        ref_m = re.match(r"q\((\d+),\s*(\d+)\)", val)
        exp.append([int(node), int(comp),
                    [int(ref_m.group(1)), int(ref_m.group(2))] if ref_m else float(val)])
    rotor = {
        "source": "tests/regression_tests/regression/iea15_rotor_data.hpp, test_rotor.cpp",
        "node_xi": node_xi,
        "node_coords": [coords[7 * i : 7 * i + 7] for i in range(len(node_xi))],
        "quadrature": [quad[2 * i : 2 * i + 2] for i in range(len(quad) // 2)],
        "sections": sections,
        "omega": [0.0, 0.0, -0.79063415025],
        "hub_radius": 3.97,
        "gravity": [-9.81, 0.0, 0.0],
        "max_iter": 6, "h": 0.01, "rho_inf": 0.0, "num_steps": 11,
        "tolerance": 1e-13,
        "expected_q": exp,
    }
    json.dump(rotor, open(os.path.join(out_dir, "iea15_rotor.json"), "w"), indent=1)

    # ---- cantilever ----------------------------------------------------------
    ct = strip_comments(open(os.path.join(reg, "test_cantilever_beam.cpp")).read())
    tips = [view_after(ct, "expect_kokkos_view_1D_equal", k) for k in range(3)]
    json.dump({"source": "tests/regression_tests/regression/test_cantilever_beam.cpp",
               "tip_q": tips, "tolerance": 1e-6},
              open(os.path.join(out_dir, "cantilever.json"), "w"), indent=1)

    # ---- solver ----------------------------------------------------------------
    st = strip_comments(open(os.path.join(reg, "test_solver.cpp")).read())
    s1 = st.index("inline void SetUpSolverAndAssemble")
    s2 = st.index("inline void SetupAndTakeNoSteps")
    s3 = st.index("inline auto SetupAndTakeTwoSteps")
    t1, t2, t3 = st[s1:s2], st[s2:s3], st[s3:]
    solver = {
        "source": "tests/regression_tests/regression/test_solver.cpp",
        "predict": {
            "residual_terms": view_after(t1, "constraints.residual_terms"),
            "b": view_after(t1, "Kokkos::subview(solver.b"),
            "q": view_after(t1, "state.q,"),
            "q_delta": view_after(t1, "state.q_delta,"),
            "v": view_after(t1, "state.v,"),
        },
        "one_iteration": {
            "x": view_after(t2, "Kokkos::subview(solver.x"),
            "convergence_err": float(re.search(r"convergence_err\[0\],\s*(" + NUM + ")",
                                               t2).group(1)),
            "q_delta": view_after(t2, "state.q_delta,"),
            "v": view_after(t2, "state.v,"),
            "vd": view_after(t2, "state.vd,"),
            "q": view_after(t2, "state.q,"),
            "lambda": view_after(t2, "constraints.lambda,"),
        },
        "two_iterations": {
            "residual_terms": view_after(t3, "constraints.residual_terms"),
            "b": view_after(t3, "Kokkos::subview(solver.b"),
            "x": view_after(t3, "Kokkos::subview(solver.x"),
        },
        "tolerance": 1e-6,
    }
    json.dump(solver, open(os.path.join(out_dir, "solver.json"), "w"), indent=1)

    # ---- rotating beam -----------------------------------------------------------
    rb = strip_comments(open(os.path.join(reg, "test_rotating_beam.cpp")).read())
    r0 = rb.index("TEST(RotatingBeamTest, StepConvergence)")
    json.dump({"source": "tests/regression_tests/regression/test_rotating_beam.cpp",
               "q": view_after(rb[r0:], "state.q,"), "tolerance": 1e-6},
              open(os.path.join(out_dir, "rotating_beam.json"), "w"), indent=1)

    # ---- rotation control (hub node, pitch about the blade axis) ------------------
    r1 = rb.index("TEST(RotatingBeamTest, RotationControlConstraint)")
    r2 = rb.index("TEST(RotatingBeamTest, CompoundRotationControlConstraint)")
    r3 = rb.index("TEST(", r2 + 5)
    rv = [float(m.group(2)) for m in
          re.finditer(r"EXPECT_NEAR\(\s*rv\[(\d)\],\s*(" + NUM + r"),\s*(" + NUM + r")\)", rb[r2:r3])]
    tol = [float(m.group(3)) for m in
           re.finditer(r"EXPECT_NEAR\(\s*rv\[(\d)\],\s*(" + NUM + r"),\s*(" + NUM + r")\)", rb[r2:r3])]
    json.dump({"source": "tests/regression_tests/regression/test_rotating_beam.cpp",
               "fixed_hub": {"steps": 10, "q": view_after(rb[r1:r2], "state.q,"), "tolerance": 1e-6},
               "prescribed_hub": {"steps": 100, "rv_root": rv, "tolerance": max(tol)}},
              open(os.path.join(out_dir, "rotation_control.json"), "w"), indent=1)

    # ---- revolute joint (ground - revolute - hub - rigid - root; generator torque) --
    j0 = rb.index("TEST(RotatingBeamTest, RevoluteJointConstraint)")
    j1 = rb.index("void GeneratorTorqueWithAxisTilt(")
    gen = {}
    for name, key in (("GeneratorTorque_Tilt0", "tilt0"), ("GeneratorTorque_Tilt90", "tilt90")):
        t0 = rb.index("TEST(RotatingBeamTest, " + name + ")")
        call = rb.index("GeneratorTorqueWithAxisTilt(", t0)
        b1 = _block(rb, call)
        p2 = rb.index(b1, call) + len(b1)
        b2 = _block(rb, p2)
        p3 = rb.index(b2, p2) + len(b2)
        b3 = _block(rb, p3)
        gen[key] = {"azimuth_q": [float(x) for x in re.findall(NUM, b1)],
                    "azimuth_v": [float(x) for x in re.findall(NUM, b2)],
                    "output": [float(x) for x in re.findall(NUM, b3)]}
    gen["tilt0"]["tilt"] = 0.0
    gen["tilt90"]["tilt"] = "pi/2"
    json.dump({"source": "tests/regression_tests/regression/test_rotating_beam.cpp",
               "revolute": {"steps": 5, "q": view_after(rb[j0:j1], "state.q,"), "tolerance": 1e-6},
               "generator_torque": dict(gen, steps=10, torque=100.0, tolerance=1e-6)},
              open(os.path.join(out_dir, "revolute_joint.json"), "w"), indent=1)

    # ---- heavy top (three-row constraints on a position-only ground node) -----------
    ht = strip_comments(open(os.path.join(reg, "test_heavy_top.cpp")).read())
    qv = [(int(m.group(1)), float(m.group(2)), float(m.group(3))) for m in
          re.finditer(r"EXPECT_NEAR\(\s*q\[0\]\[(\d)\],\s*(" + NUM + r"),\s*(" + NUM + r")\)", ht)]
    json.dump({"source": "tests/regression_tests/regression/test_heavy_top.cpp",
               "steps": 400, "q_mass_node": [v for _, v, _ in sorted(qv)],
               "tolerance": max(t for _, _, t in qv)},
              open(os.path.join(out_dir, "heavy_top.json"), "w"), indent=1)

    # ---- CFD interface: floating platform (mass + mooring springs, three-row constraints)
    cf = strip_comments(open(os.path.join(ref, "tests", "regression_tests", "interfaces",
                                          "test_cfd_interface.cpp")).read())
    c0 = cf.index("TEST(CFDInterfaceTest, PrecessionTest)")
    c1 = cf.index("TEST(CFDInterfaceTest, FloatingPlatform)")
    c2 = cf.index("TEST(CFDInterfaceTest, Restart)")
    pat = r"EXPECT_NEAR\(\s*platform_node\.displacement\[(\d)\],\s*(" + NUM + r"),\s*(" + NUM + r")\)"
    pre = [(int(m.group(1)), float(m.group(2)), float(m.group(3))) for m in re.finditer(pat, cf[c0:c1])]
    pat2 = r"EXPECT_NEAR\(\s*platform_u\[(\d)\],\s*(" + NUM + r"),\s*(" + NUM + r")\)"
    fpl = [(int(m.group(1)), float(m.group(2)), float(m.group(3))) for m in re.finditer(pat2, cf[c1:c2])]
    json.dump({"source": "tests/regression_tests/interfaces/test_cfd_interface.cpp",
               "precession": {"q_500": [v for _, v, _ in pre[0:7]], "q_600": [v for _, v, _ in pre[7:14]],
                              "tolerance": max(t for _, _, t in pre)},
               "floating_platform": {"step": 100, "q": [v for _, v, _ in fpl],
                                     "tolerance": max(t for _, _, t in fpl)}},
              open(os.path.join(out_dir, "cfd_platform.json"), "w"), indent=1)

    # ---- revolute joint kernels (unit tests: residual/gradients, torque, output) ----
    ut = os.path.join(ref, "tests", "unit_tests", "constraints")

    def views(text):
        out = {}
        for mm in re.finditer(r'CreateView<[^>]*>\(\s*"(\w+)",\s*std::array(?:<[^>]*>)?\{', text):
            out[mm.group(1)] = [float(x) for x in re.findall(NUM, _block(text, mm.end() - 1))]
        for mm in re.finditer(r"(\w+_exact_data)\s*=\s*std::array\{", text):
            out[mm.group(1)] = [float(x) for x in re.findall(NUM, _block(text, mm.end() - 1))]
        return out
    rj = {}
    for key, fname in (("constraint", "test_calculate_revolute_joint_constraint.cpp"),
                       ("force", "test_calculate_revolute_joint_force.cpp"),
                       ("output", "test_calculate_revolute_joint_output.cpp")):
        rj[key] = views(strip_comments(open(os.path.join(ut, fname)).read()))
    rj["source"] = "tests/unit_tests/constraints/test_calculate_revolute_joint_{constraint,force,output}.cpp"
    rj["tolerance"] = 1e-15
    json.dump(rj, open(os.path.join(out_dir, "revolute_unit.json"), "w"), indent=1)
    cu = {}
    for key, fname in (("fixed_bc", "test_calculate_fixed_bc_constraint.cpp"),
                       ("prescribed_bc", "test_calculate_prescribed_bc_constraint.cpp"),
                       ("rigid_joint", "test_calculate_rigid_joint_constraint.cpp"),
                       ("rotation_control", "test_calculate_rotation_control_constraint.cpp")):
        cu[key] = views(strip_comments(open(os.path.join(ut, fname)).read()))
    cu["source"] = "tests/unit_tests/constraints/test_calculate_{fixed_bc,prescribed_bc,rigid_joint,rotation_control}_constraint.cpp"
    json.dump(cu, open(os.path.join(out_dir, "constraint_unit.json"), "w"), indent=1)

    # ---- point masses and springs -------------------------------------------------
    def near_calls(text: str, name: str):
        pat = (r"EXPECT_NEAR\(\s*" + name + r"\((\d+),\s*(\d+)\),\s*(" + NUM + r"),\s*(" + NUM +
               r")\s*\)")
        return [(int(m.group(1)), int(m.group(2)), float(m.group(3)), float(m.group(4)))
                for m in re.finditer(pat, text)]
    ms = strip_comments(open(os.path.join(reg, "test_masses.cpp")).read())
    ms = ms[ms.index("TEST(MassesTest, ExternalForce)"):]
    pr = strip_comments(open(os.path.join(reg, "test_precession.cpp")).read())
    sm = strip_comments(open(os.path.join(reg, "test_spring_mass_system.cpp")).read())
    s1 = sm.index("SetUpSpringMassSystem()")
    s2 = sm.index("SetUpSpringMassChainSystem()")
    half, full = near_calls(sm[s1:s2], "q")[1], near_calls(sm[s1:s2], "q")[3]
    json.dump({"source": ["tests/regression_tests/regression/test_masses.cpp",
                          "tests/regression_tests/regression/test_precession.cpp",
                          "tests/regression_tests/regression/test_spring_mass_system.cpp"],
               "mass_external_force": {"steps": 1000, "v": [c[2] for c in near_calls(ms, "v_host")],
                                       "tolerance": max(c[3] for c in near_calls(ms, "v_host"))},
               "precession": {"steps": 500, "q": [c[2] for c in near_calls(pr, "q_host")],
                              "tolerance": max(c[3] for c in near_calls(pr, "q_host"))},
               "spring_mass": {"steps": 1000, "q1x_half": half[2], "q1x_end": full[2],
                               "tolerance": max(half[3], full[3])},
               "spring_mass_chain": {"steps": 1000, "tolerance": 1e-14}},
              open(os.path.join(out_dir, "masses_springs.json"), "w"), indent=1)

    # ---- IEA-15 blade through the blade interface (WindIO input) ----------------
    # tests/regression_tests/interfaces/test_blade_interface.cpp:13-128 reads the
    # WindIO file of interfaces_test_files; its blade axis, twist and 6x6 section
    # tables go to a plain-number file the C++ driver reads, with the expected
    # tip position of the test.
    import yaml
    itf = os.path.join(ref, "tests", "regression_tests", "interfaces")
    wio = yaml.safe_load(open(os.path.join(itf, "interfaces_test_files", "IEA-15-240-RWT.yaml")))
    bl = wio["components"]["blade"]
    ra = bl["outer_shape_bem"]["reference_axis"]
    tw = bl["outer_shape_bem"]["twist"]
    kk = bl["elastic_properties_mb"]["six_x_six"]["stiff_matrix"]
    mm = bl["elastic_properties_mb"]["six_x_six"]["inertia_matrix"]
    bt = strip_comments(open(os.path.join(itf, "test_blade_interface.cpp")).read())
    b0 = bt.index("TEST(BladeInterfaceTest, BladeWindIO)")
    b1 = bt.index("TEST(", b0 + 5)
    tip = [float(m.group(2)) for m in
           re.finditer(r"EXPECT_NEAR\(\s*tip_node\.position\[(\d)\],\s*(" + NUM + r"),", bt[b0:b1])]
    assert len(tip) == 7
    lines = [str(len(ra["x"]["grid"]))]
    for i, g in enumerate(ra["x"]["grid"]):
        lines.append(" ".join(repr(float(v)) for v in (g, ra["x"]["values"][i], ra["y"]["values"][i],
                                                        ra["z"]["values"][i])))
    lines.append(str(len(tw["grid"])))
    for g, v in zip(tw["grid"], tw["values"]):
        lines.append(f"{float(g)!r} {float(v)!r}")
    lines.append(str(len(kk["grid"])))
    for i, g in enumerate(kk["grid"]):
        assert abs(mm["grid"][i] - g) <= 1e-8
        lines.append(" ".join(repr(float(v)) for v in [g] + list(mm["values"][i]) + list(kk["values"][i])))
    lines.append(" ".join(repr(v) for v in tip))
    with open(os.path.join(out_dir, "iea15_blade_windio.txt"), "w") as f:
        f.write("# IEA-15-240-RWT blade (WindIO) for BladeInterfaceTest.BladeWindIO:\n"
                "# axis points (grid x y z), twist (grid deg), sections (grid inertia[21] stiffness[21]),\n"
                "# expected tip position [7]\n" + "\n".join(lines) + "\n")

    # ---- IEA-15 turbine through the turbine interface (WindIO input) ----------------
    # tests/regression_tests/interfaces/test_turbine_interface.cpp:17-285 builds
    # the whole turbine from the same WindIO file: the blade input above, the
    # tower (reference axis, outer diameter and wall thickness of its first
    # layer, isotropic material), the hub and the nacelle; the expected tower
    # top position of the test closes the file.
    tt = strip_comments(open(os.path.join(itf, "test_turbine_interface.cpp")).read())
    t0 = tt.index("TEST(TurbineInterfaceTest, IEA15_Structure)")
    top = [float(m.group(2)) for m in
           re.finditer(r"EXPECT_NEAR\(\s*tower_top_node\.position\[(\d)\],\s*(" + NUM + r"),", tt[t0:])]
    assert len(top) == 7
    tower = wio["components"]["tower"]
    tra = tower["outer_shape_bem"]["reference_axis"]
    tdia = tower["outer_shape_bem"]["outer_diameter"]
    layer = tower["internal_structure_2d_fem"]["layers"][0]
    mat = next(m for m in wio["materials"] if m.get("name") == layer["material"])
    hub = wio["components"]["hub"]
    nac = wio["components"]["nacelle"]
    tl = [str(len(tra["x"]["grid"]))]
    for i, g in enumerate(tra["x"]["grid"]):
        tl.append(" ".join(repr(float(v)) for v in (g, tra["x"]["values"][i], tra["y"]["values"][i],
                                                     tra["z"]["values"][i])))
    tl.append(str(len(tdia["grid"])))
    for i, g in enumerate(tdia["grid"]):
        tl.append(" ".join(repr(float(v)) for v in (g, tdia["values"][i], layer["thickness"]["values"][i])))
    tl.append(" ".join(repr(float(mat[k])) for k in ("E", "G", "rho", "nu")))
    tl.append(" ".join(repr(float(v)) for v in [hub["diameter"], hub["cone_angle"],
                                                  hub["elastic_properties_mb"]["system_mass"]]
                       + list(hub["elastic_properties_mb"]["system_inertia"])))
    dt = nac["drivetrain"]
    ep = nac["elastic_properties_mb"]
    tl.append(" ".join(repr(float(v)) for v in [dt["uptilt"], dt["overhang"], dt["distance_tt_hub"],
                                                  ep["system_mass"], ep["yaw_mass"]]
                       + list(ep["system_inertia_tt"])))
    tl.append(" ".join(repr(v) for v in top))
    with open(os.path.join(out_dir, "iea15_turbine_windio.txt"), "w") as f:
        f.write("# IEA-15-240-RWT tower, hub and nacelle (WindIO) for TurbineInterfaceTest.IEA15_Structure\n"
                "# (the blades use iea15_blade_windio.txt): tower axis points (grid x y z), tower stations\n"
                "# (grid outer_diameter wall_thickness), tower material (E G rho nu), hub (diameter\n"
                "# cone_angle mass inertia[6]), nacelle (uptilt overhang distance_tt_hub system_mass\n"
                "# yaw_mass inertia_tt[6]), expected tower top position [7]\n" + "\n".join(tl) + "\n")

    # ---- curved beam (kernel level) --------------------------------------------
    cb = strip_comments(open(os.path.join(unit, "test_curved_beam.hpp")).read())
    names = ["kCurvedBeamNodes_data", "kGaussQuadraturePoints", "kGaussQuadratureWeights",
             "kExpectedInterpWeights", "kExpectedDerivWeights", "kExpectedJacobians",
             "kCurvedBeamCuu_data", "kCurvedBeamStrain_data", "kExpectedFc_data",
             "kX0pupSS_data", "kExpectedFd_data", "kInterpWeightsFlat", "kDerivWeightsFlat",
             "kFc", "kFd", "kFi", "kExpectedResidualVector", "xr_data", "Cstar_data",
             "kExpectedCuu_data", "kCurvedBeamM_tilde_data", "kCurvedBeamN_tilde_data",
             "kExpectedOuu_data", "kExpectedPuu_data", "kExpectedQuu_data", "kKuu", "kOuu",
             "kPuu", "kQuu", "kCuu", "kExpectedStiffnessMatrix_data"]
    curved = {"source": "tests/unit_tests/system/beams/test_curved_beam.hpp"}
    known = {"kStrainInterpolationHolder": numbers_of(cb, "kStrainInterpolationHolder")}
    for n in names:
        curved[n] = numbers_of(cb, n, known)
    ctcpp = open(os.path.join(unit, "test_curved_beam.cpp")).read()
    gll = re.search(r"kGLLNodes\s*\{([^}]*)\}", cb)
    curved["kGLLNodes"] = [float(x) for x in re.findall(NUM, gll.group(1))]
    curved["tolerance"] = 1e-12
    curved["test_source_lines"] = len(ctcpp.splitlines())
    json.dump(curved, open(os.path.join(out_dir, "curved_beam.json"), "w"), indent=1)
    print("wrote fixtures to", out_dir)


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("KYN_REFERENCE_ROOT")
    if not root:
        sys.exit("usage: make_golden.py <reference root>  (or set KYN_REFERENCE_ROOT)")
    main(root)
