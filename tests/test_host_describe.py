"""Host-side model setup without a GPU (kyn_model_describe): every model type
the path accepts gets the reference's DOF counts and CRS graph (compared with
the oracle's, which follows src/solver/create_full_matrix.hpp), and the
topologies outside the path are refused with KYN_ERR_UNSUPPORTED."""
import math

import numpy as np
import pytest

from openturbine_b200 import workloads as W
from openturbine_b200.model import BeamSection, Model
from openturbine_b200.runtime import describe
from oracle.oracle_py import OracleModel
from tests import workloads_ref as R


def _first(x):
    return x[0] if isinstance(x, tuple) else x


MODELS = {
    "cantilever": lambda: R.cantilever_test_model(),
    "solver": lambda: R.solver_test_model(),
    "rotating_beam": lambda: R.rotating_beam_test_model(),
    "iea15_rotor": lambda: R.iea15_rotor_model(),
    "iea15_hub_rotor": lambda: R.iea15_hub_rotor_model(),
    "rotation_control_fixed_hub": lambda: R.rotation_control_test_model(False),
    "rotation_control_prescribed_hub": lambda: R.rotation_control_test_model(True),
    "revolute_ground_hub": lambda: R.revolute_joint_test_model(),
    "generator_torque_tilt0": lambda: R.generator_torque_model(0.0),
    "generator_torque_tilt90": lambda: R.generator_torque_model(math.pi / 2.),
    "heavy_top": lambda: R.heavy_top_model(),
    "cfd_spinning_platform": lambda: R.cfd_platform_model(False),
    "cfd_moored_platform": lambda: R.cfd_platform_model(True),
    "mass_external_force": lambda: R.mass_external_force_model(),
    "precession": lambda: R.precession_model(),
    "spring_mass": lambda: R.spring_mass_model(),
    "spring_mass_chain": lambda: R.spring_mass_chain_model(),
    "two_element_cantilever": lambda: R.two_element_cantilever_model(),
    "two_beams_rigid_joint": lambda: R.two_beams_model(),
    "moored_cantilever": lambda: R.moored_cantilever_model(),
    "condensed_four_element_cantilever": lambda: R.four_element_cantilever_model(),
    "condensed_tower": lambda: R.tower_model(),
    "condensed_two_long_beams": lambda: R.two_long_beams_model(),
    "dense_revolute_pendulum": lambda: R.revolute_pendulum_model(),
    "three_row_bc_on_a_beam": lambda: _cantilever_with(lambda m: m.AddFixedBC3DOFs(4)),
    "batch_rotor": lambda: W.rotor_model(3),
    "batch_cantilever": lambda: W.batch_cantilever_model(W.draw_batch(1, first_id=77)[0]),
}


@pytest.mark.parametrize("name", sorted(MODELS))
def test_dofs_and_crs_graph_match_the_oracle(name):
    pm = _first(MODELS[name]()).pack()
    info, rp, ci = describe(pm)
    o = OracleModel(pm)
    orp, oci, _ = o.crs()
    assert (info.num_dofs, info.num_system_dofs, info.nnz) == (o.info.num_dofs, o.info.num_system_dofs,
                                                                o.info.nnz)
    assert np.array_equal(rp, orp) and np.array_equal(ci, oci)
    assert info.device_bytes > 0


def _cantilever_with(extra):
    m = R.cantilever_test_model()[0]
    extra(m)
    return m


def _two_revolute_joints():
    m = R.generator_torque_model(0.0)[0]
    n = m.AddNode().SetPosition(0., 0., 5., 1., 0., 0., 0.).Build()
    m.AddMassElement(n, np.eye(6))
    m.AddRevoluteJointConstraint([len(m.nodes_) - 4, n], [0., 0., 1.], np.zeros(1))
    return m


def _revolute_in_a_dense_model():
    m = R.heavy_top_model()[0]
    n = m.AddNode().SetPosition(0., 2., 0., 1., 0., 0., 0.).Build()
    m.AddMassElement(n, np.eye(6))
    m.AddRevoluteJointConstraint([0, n], [0., 0., 1.], np.zeros(1))
    return m


# Revolute joints outside a drive train (a second joint, a joint between beam
# nodes, a joint in a beam-free dense model) make the model a dense bordered
# system, where each revolute joint is five constraint rows.
MODELS.update({
    "two_revolute_joints": _two_revolute_joints,
    "revolute_between_beam_nodes": lambda: _cantilever_with(
        lambda m: m.AddRevoluteJointConstraint([1, 2], [1., 0., 0.], np.zeros(1))),
    "revolute_in_a_dense_model": _revolute_in_a_dense_model,
})


@pytest.mark.parametrize("name", ["two_revolute_joints", "revolute_between_beam_nodes",
                                  "revolute_in_a_dense_model"])
def test_revolute_joints_outside_a_drive_train_go_dense(name):
    pm = _first(MODELS[name]()).pack()
    info, rp, ci = describe(pm)
    o = OracleModel(pm)
    orp, oci, _ = o.crs()
    assert info.num_dofs == o.info.num_dofs
    assert np.array_equal(rp, orp) and np.array_equal(ci, oci)


@pytest.mark.parametrize("case", ["free_node_outside_the_beams", "seventeen_constraints_in_a_dense_model"])
def test_topologies_outside_the_path_are_refused(case):
    if case == "seventeen_constraints_in_a_dense_model":
        m = R.heavy_top_model()[0]
        for k in range(17):
            n = m.AddNode().SetPosition(0., 2. + k, 0., 1., 0., 0., 0.).Build()
            m.AddMassElement(n, np.eye(6))
            m.AddRigidJointConstraint([0, n])
    else:
        m = _cantilever_with(lambda m: m.AddNode().SetPosition(0., 5., 0., 1., 0., 0., 0.).Build())
    with pytest.raises(RuntimeError, match="UNSUPPORTED"):
        describe(m.pack())
