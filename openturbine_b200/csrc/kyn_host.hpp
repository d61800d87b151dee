// kyn_host.hpp -- host-side model setup for the B200 beam path.
//
// Turns a kyn_model_desc into per-beam slabs (constant geometry plus initial
// state, see SlabLayout) and the reference's CRS graph of the model.  This is
// the once-per-model work that Model::CreateSystemWithSolver does on the host
// and in setup kernels (src/model/model.hpp:42-63, 647-656;
// src/elements/beams/create_beams.hpp:27-165; src/dof_management/*;
// src/solver/create_full_matrix.hpp:27-73).
#pragma once

#include <string>
#include <vector>

#include "../../include/kynema_b200.h"
#include "kyn_types.h"

namespace kyn {

// One CTA's system: a beam element, or several elements sharing nodes (a
// multi-element beam), or the nodes of a model without beam elements.
struct HostBeam {
    int N = 0, Q = 0, nc = 0;
    std::vector<int> node_ids;        // global node ids (local node order)
    std::vector<int> elem_ids;        // beam elements in this system (model order)
    std::vector<std::vector<int>> elem_local;  // local index of each element node
    std::vector<double> slab;         // SlabLayout-ordered doubles
    int con_node[kMaxBeamConstraints] = {};
    int con_type[kMaxBeamConstraints] = {};
    int con_row[kMaxBeamConstraints] = {};   // constraint index in the model
    double con_X0[kMaxBeamConstraints][3] = {};
    double con_axis[kMaxBeamConstraints][3] = {};  // RotationControl: unit axis
    bool lumped = false;              // all nodes of a model without beam elements (Q = 0)
    bool dense = false;               // solved as the dense bordered system (one CTA, pivoted LU)
    int n_comps = 0;                  // dense model with beams: beam components in the slab
    int comps_off = 0;                // their header's offset in the slab (kCompHead records)
    int comp_maxN = 0, comp_maxQ = 0; // largest component
    int con_base[kMaxBeamConstraints] = {-1, -1, -1, -1, -1, -1, -1, -1,
                                         -1, -1, -1, -1, -1, -1, -1, -1};  // dense: joint base (local)
    int cond_nd = 0;                  // condensed dense model: bordered-system unknowns, else 0
    int cond_md_off = -1;             // offset of that system in the slab when it lives in device memory
    int frames_off = -1;              // dense model with revolute joints: [nc][9] joint frames in the slab
    int n_mass = 0, n_spring = 0;     // point masses / springs at this beam's nodes
    int lumped_off = 0;               // their records' offset in the slab (kMassRec, kSpringRec)
};

struct HostModel {
    int num_nodes = 0;
    int num_elements = 0;                     // beam elements of the description
    std::vector<int> elem_row;                // first node_FX row of each element
    int num_constraints = 0;
    std::vector<HostBeam> beams;
    std::vector<int> node_beam, node_local;   // node -> (beam, local index)
    std::vector<int> con_beam, con_slot;      // constraint -> (beam, slot)
    std::vector<int> spring_nodes;            // [springs][2] global node ids
    std::vector<int> fmap;                    // node -> first DOF
    std::vector<int> active;                  // node -> DOFs (6, or 3 for position-only nodes)
    int nsys = 0, ndofs = 0;
    std::vector<int> row_ptrs, col_inds;      // reference CRS graph (sorted rows)
    double gravity[3] = {0., 0., 0.};
    int hub = -1;                             // hub node (in no beam) or -1
    int hub_con = -1;                         // the single-node BC holding the hub
    int hub_con_type = 0;
    // Drive train: the hub chain (hubrec records 0..): shaft base (= hub, held
    // by hub_con), revolute target, optional node rigidly jointed to it.  A
    // plain hub is a chain of one.  The beam roots join chain.back().
    std::vector<int> chain;
    int rev_con = -1;                         // the revolute joint (chain 0 -> 1)
    int ah_con = -1;                          // the rigid joint chain 1 -> 2, or -1
    std::vector<int> con_row_first;           // constraint -> first row (after nsys)
    std::vector<int> con_rows;                // constraint -> rows (5 revolute, else 6)
};

// Validates the description and builds the host model.  Returns KYN_OK or a
// negative KYN_ERR_* code with a message in `err`.
int build_host_model(const kyn_model_desc* d, HostModel& out, std::string& err);

// Lagrange basis on nodes xs evaluated at x: values and first derivatives.
void lagrange_basis(double x, const std::vector<double>& xs, std::vector<double>& val,
                    std::vector<double>& der);

}  // namespace kyn
