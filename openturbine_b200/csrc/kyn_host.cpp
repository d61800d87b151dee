// kyn_host.cpp -- host-side model setup for the B200 beam path (see kyn_host.hpp).
#include "kyn_host.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>

namespace kyn {

namespace {

// Hamilton product and rotation of a vector (src/math/quaternion_operations.hpp).
void qmul(const double* a, const double* b, double* o) {
    o[0] = a[0] * b[0] - a[1] * b[1] - a[2] * b[2] - a[3] * b[3];
    o[1] = a[0] * b[1] + a[1] * b[0] + a[2] * b[3] - a[3] * b[2];
    o[2] = a[0] * b[2] - a[1] * b[3] + a[2] * b[0] + a[3] * b[1];
    o[3] = a[0] * b[3] + a[1] * b[2] - a[2] * b[1] + a[3] * b[0];
}

int fail(std::string& err, int code, const char* msg) {
    err = msg;
    return code;
}

}  // namespace

void lagrange_basis(double x, const std::vector<double>& xs, std::vector<double>& val,
                    std::vector<double>& der) {
    // l_i(x) = prod_{m != i} (x - x_m) / (x_i - x_m)
    // l_i'(x) = sum_{j != i} 1/(x_i - x_j) prod_{k != i,j} (x - x_k)/(x_i - x_k)
    // (src/math/interpolation.hpp LagrangePolynomial{Interp,Deriv}Weights)
    const size_t n = xs.size();
    val.assign(n, 1.);
    der.assign(n, 0.);
    for (size_t i = 0; i < n; ++i) {
        for (size_t m = 0; m < n; ++m)
            if (m != i) val[i] *= (x - xs[m]) / (xs[i] - xs[m]);
        double d = 0.;
        for (size_t j = 0; j < n; ++j) {
            if (j == i) continue;
            double p = 1.;
            for (size_t k = 0; k < n; ++k)
                if (k != i && k != j) p *= (x - xs[k]) / (xs[i] - xs[k]);
            d += p / (xs[i] - xs[j]);
        }
        der[i] = d;
    }
}

// Node state of a beam's (or a lumped model's) slab from the description
// (src/model/copy_nodes_to_state.hpp:14-60).
// Shape tables, quadrature weights, Jacobian, reference line tangent, r0 and
// interpolated sections of element e's quadrature points, written at points
// [qo, qo + Q_e) of a slab over N local nodes; element node k is local column
// loc[k] (global node enode[k]).
static int fill_element_qps(const kyn_model_desc* d, int e, const std::vector<int>& enode,
                            const std::vector<int>& loc, int Nloc, int qo, const SlabLayout& L,
                            double* S, std::string& err) {
    const int s0 = d->beam_section_offsets[e], s1 = d->beam_section_offsets[e + 1];
    const int q0 = d->beam_qp_offsets[e], q1 = d->beam_qp_offsets[e + 1];
    const int N = static_cast<int>(enode.size()), Q = q1 - q0;
    // shape functions on node locations xi = 2 s - 1 (populate_element_views.hpp:45-78)
    std::vector<double> node_xi(N), val, der;
    for (int k = 0; k < N; ++k) node_xi[k] = 2. * d->node_s[enode[k]] - 1.;
    for (int a = 0; a < N; ++a)
        for (int b = a + 1; b < N; ++b)
            if (node_xi[a] == node_xi[b])
                return fail(err, KYN_ERR_INVALID, "two beam nodes share an element location");
    std::vector<double> sec_xi(s1 - s0);
    for (int s = s0; s < s1; ++s) sec_xi[s - s0] = 2. * d->section_position[s] - 1.;
    for (int q = 0; q < Q; ++q) {
        const double xi = d->qp_xi[q0 + q];
        lagrange_basis(xi, node_xi, val, der);
        for (int k = 0; k < N; ++k) {
            S[L.phi + (qo + q) * Nloc + loc[k]] = val[k];
            S[L.dphi + (qo + q) * Nloc + loc[k]] = der[k];
        }
        // sections: linear interpolation in xi, clamped at the ends
        // (populate_element_views.hpp:90-141, interpolation.hpp LinearInterpWeights)
        std::vector<double> wsec(sec_xi.size(), 0.);
        const auto lo = std::lower_bound(sec_xi.begin(), sec_xi.end(), xi);
        if (lo == sec_xi.begin()) {
            wsec.front() = 1.;
        } else if (lo == sec_xi.end()) {
            wsec.back() = 1.;
        } else {
            const size_t idx = static_cast<size_t>(lo - sec_xi.begin());
            const double wu = (xi - sec_xi[idx - 1]) / (sec_xi[idx] - sec_xi[idx - 1]);
            wsec[idx - 1] = 1. - wu;
            wsec[idx] = wu;
        }
        for (int k = 0; k < 36; ++k) {
            double m = 0., c = 0.;
            for (size_t s = 0; s < sec_xi.size(); ++s) {
                m += d->section_mass[(s0 + s) * 36 + k] * wsec[s];
                c += d->section_stiffness[(s0 + s) * 36 + k] * wsec[s];
            }
            S[L.mstar + (qo + q) * 36 + k] = m;
            S[L.cstar + (qo + q) * 36 + k] = c;
        }
        // reference rotation: normalised interpolated node orientation
        // (interpolation_operations.hpp InterpQuaternion)
        double r[4] = {0., 0., 0., 0.};
        double xp[3] = {0., 0., 0.};
        for (int k = 0; k < N; ++k) {
            const double* x0 = d->node_x0 + enode[k] * 7;
            for (int c = 0; c < 4; ++c) r[c] += x0[3 + c] * val[k];
            for (int c = 0; c < 3; ++c) xp[c] += x0[c] * der[k];
        }
        const double rl = std::sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2] + r[3] * r[3]);
        if (rl == 0.) {
            S[L.r0 + (qo + q) * 4] = 1.;
        } else {
            for (int c = 0; c < 4; ++c) S[L.r0 + (qo + q) * 4 + c] = r[c] / rl;
        }
        // Jacobian |dx0/dxi| and unit tangent (calculate_jacobian.hpp:36-76)
        const double J = std::sqrt(xp[0] * xp[0] + xp[1] * xp[1] + xp[2] * xp[2]);
        if (!(J > 0.)) return fail(err, KYN_ERR_INVALID, "degenerate beam reference line");
        for (int c = 0; c < 3; ++c) S[L.x0p + (qo + q) * 3 + c] = xp[c] / J;
        const double w = d->qp_weight[q0 + q];
        for (int k = 0; k < N; ++k)
            S[L.dphiJ + (qo + q) * Nloc + loc[k]] = S[L.dphi + (qo + q) * Nloc + loc[k]] / J;
        S[L.qpw + (qo + q) * 4 + 0] = w;
        S[L.qpw + (qo + q) * 4 + 1] = J;
        S[L.qpw + (qo + q) * 4 + 2] = w * J;
        S[L.qpw + (qo + q) * 4 + 3] = w / J;
    }
    return KYN_OK;
}

static void init_node_state(const kyn_model_desc* d, const HostBeam& B, const SlabLayout& L,
                            double* S) {
    static const double ident[7] = {0., 0., 0., 1., 0., 0., 0.};
    for (int k = 0; k < B.N; ++k) {
        const int id = B.node_ids[k];
        const double* x0 = d->node_x0 + id * 7;
        const double* u = d->node_u ? d->node_u + id * 7 : ident;
        for (int c = 0; c < 7; ++c) {
            S[L.x0 + k * 7 + c] = x0[c];
            S[L.q + k * 7 + c] = u[c];
            S[L.q_prev + k * 7 + c] = u[c];
        }
        for (int c = 0; c < 3; ++c) S[L.x + k * 7 + c] = x0[c] + u[c];
        qmul(u + 3, x0 + 3, S + L.x + k * 7 + 3);
        for (int c = 0; c < 6; ++c) {
            S[L.v + k * 6 + c] = d->node_v ? d->node_v[id * 6 + c] : 0.;
            S[L.vd + k * 6 + c] = d->node_vd ? d->node_vd[id * 6 + c] : 0.;
            S[L.a + k * 6 + c] = S[L.vd + k * 6 + c];
        }
        for (int c = 0; c < 3; ++c) S[L.tangent + k * 9 + c * 4] = 1.;
    }
}

// Frame of a revolute joint (src/constraints/constraints.hpp:294-319): x_hat =
// unit(axis), or unit(X0) for a zero axis; the rows of the rotation taking
// (1, 0, 0) to x_hat are the joint axes x0, y0, z0.
static int revolute_frame(const double* ax, const double X0[3], double axes[9], std::string& err) {
    const double na = ax ? std::sqrt(ax[0] * ax[0] + ax[1] * ax[1] + ax[2] * ax[2]) : 0.;
    const double* src = na != 0. ? ax : X0;
    const double ns = std::sqrt(src[0] * src[0] + src[1] * src[1] + src[2] * src[2]);
    if (!(ns > 0.)) return fail(err, KYN_ERR_INVALID, "revolute joint needs an axis or distinct node positions");
    const double xh[3] = {src[0] / ns, src[1] / ns, src[2] / ns};
    const double cp[3] = {0., -xh[2], xh[1]};
    const double dp = xh[0];
    if (!(1. + dp > 0.)) return fail(err, KYN_ERR_UNSUPPORTED, "revolute joint axis along -x");
    const double kk = 1. / (1. + dp);
    const double R[9] = {cp[0] * cp[0] * kk + dp, cp[1] * cp[0] * kk + cp[2], cp[2] * cp[0] * kk - cp[1],
                         cp[0] * cp[1] * kk - cp[2], cp[1] * cp[1] * kk + dp, cp[2] * cp[1] * kk + cp[0],
                         cp[0] * cp[2] * kk + cp[1], cp[1] * cp[2] * kk - cp[0], cp[2] * cp[2] * kk + dp};
    for (int k = 0; k < 9; ++k) axes[k] = R[k];
    return KYN_OK;
}

// A model with beam elements whose constraints the per-beam systems cannot
// take: three-row constraints, a joint whose base node is a beam node (beams
// coupled to each other, a beam carrying a position-only node), or more than
// one revolute joint (the per-beam systems take one, in a drive train).
static bool needs_dense_beams(const kyn_model_desc* d) {
    if (d->num_beams <= 0 || d->num_constraints <= 0 || !d->constraint_type) return false;
    std::vector<char> in_beam(d->num_nodes, 0);
    for (int k = 0; k < d->beam_node_offsets[d->num_beams]; ++k) {
        const int id = d->beam_node_ids[k];
        if (id >= 0 && id < d->num_nodes) in_beam[id] = 1;
    }
    int revolute = 0;
    for (int c = 0; c < d->num_constraints; ++c) {
        const int t = d->constraint_type[c];
        const int base = d->constraint_base_node ? d->constraint_base_node[c] : -1;
        if (t >= KYN_CONSTRAINT_FIXED_BC_3DOF) return true;
        if ((is_hub_joint(t) || t == KYN_CONSTRAINT_RIGID_JOINT_6DOF_TO_3DOF || t == KYN_CONSTRAINT_REVOLUTE_JOINT) &&
            base >= 0 && base < d->num_nodes && in_beam[base])
            return true;
        revolute += t == KYN_CONSTRAINT_REVOLUTE_JOINT;
    }
    return revolute > 1;
}

// FreedomSignature bits of every node in a dense model
// (assemble_node_freedom_allocation_table.hpp): masses and six-row
// constraints all six components, springs and three-row constraints the
// positions; with_beams adds the beam nodes (all six).  Out-of-range ids are
// skipped (the model is validated elsewhere).
static std::vector<int> node_signatures(const kyn_model_desc* d, bool with_beams) {
    const int nn = d->num_nodes;
    std::vector<int> sig(nn, 0);
    auto set = [&](int n, int bits) {
        if (n >= 0 && n < nn) sig[n] |= bits;
    };
    for (int e = 0; e < d->num_masses && d->mass_node; ++e) set(d->mass_node[e], kSigAll);
    for (int e = 0; e < d->num_springs && d->spring_nodes; ++e) {
        set(d->spring_nodes[2 * e], kSigPosition);
        set(d->spring_nodes[2 * e + 1], kSigPosition);
    }
    for (int c = 0; c < d->num_constraints && d->constraint_type && d->constraint_target_node; ++c) {
        const int t = d->constraint_type[c];
        set(d->constraint_target_node[c], t >= KYN_CONSTRAINT_FIXED_BC_3DOF ? kSigPosition : kSigAll);
        if ((is_hub_joint(t) || t == KYN_CONSTRAINT_RIGID_JOINT_6DOF_TO_3DOF || t == KYN_CONSTRAINT_REVOLUTE_JOINT) &&
            d->constraint_base_node)
            set(d->constraint_base_node[c], kSigAll);
    }
    for (int k = 0; with_beams && d->num_beams > 0 && k < d->beam_node_offsets[d->num_beams]; ++k)
        set(d->beam_node_ids[k], kSigAll);
    return sig;
}

// Unknowns of the dense bordered system over all nodes and constraint rows.
static int dense_unknowns(const kyn_model_desc* d, bool with_beams) {
    int n = 0;
    for (int s : node_signatures(d, with_beams)) n += s == kSigAll ? 6 : s == kSigPosition ? 3 : 0;
    for (int c = 0; c < d->num_constraints && d->constraint_type; ++c) n += constraint_rows(d->constraint_type[c]);
    return n;
}

int build_host_model(const kyn_model_desc* d, HostModel& M, std::string& err) {
    if (!d) return fail(err, KYN_ERR_INVALID, "null model description");
    if (d->num_nodes <= 0 || !d->node_x0 || !d->node_s)
        return fail(err, KYN_ERR_INVALID, "model needs nodes with x0 and s");
    const int n_mass = d->num_masses > 0 ? d->num_masses : 0;
    const int n_spring = d->num_springs > 0 ? d->num_springs : 0;
    if ((n_mass > 0 && (!d->mass_node || !d->mass_matrix)) ||
        (n_spring > 0 && (!d->spring_nodes || !d->spring_stiffness || !d->spring_length)))
        return fail(err, KYN_ERR_INVALID, "mass or spring arrays missing");
    // A model without beam elements is a lumped model: its masses, springs and
    // boundary conditions form one dense system over all its nodes.
    const bool lumped = d->num_beams == 0;
    if (lumped && n_mass + n_spring == 0)
        return fail(err, KYN_ERR_INVALID, "model needs beam elements, point masses or springs");
    if (!lumped && (d->num_beams < 0 || !d->beam_node_offsets || !d->beam_node_ids ||
                    !d->beam_section_offsets || !d->beam_qp_offsets || !d->section_position ||
                    !d->section_mass || !d->section_stiffness || !d->qp_xi || !d->qp_weight))
        return fail(err, KYN_ERR_INVALID, "model needs at least one fully described beam");
    if (lumped && d->num_nodes > KYN_LUMPED_MAX_NODES)
        return fail(err, KYN_ERR_UNSUPPORTED, "lumped model larger than KYN_LUMPED_MAX_NODES nodes");
    if (d->num_beams > kMaxClusterBeams)
        return fail(err, KYN_ERR_UNSUPPORTED, "more than 8 beam elements in one model");
    const int nn = d->num_nodes;
    M.num_nodes = nn;
    M.num_constraints = d->num_constraints;
    for (int c = 0; c < 3; ++c) M.gravity[c] = d->gravity[c];
    M.node_beam.assign(nn, -1);
    M.node_local.assign(nn, -1);
    // Elements that share nodes form one system (a multi-element beam): group
    // them into connected components; each component is one CTA's system over
    // its nodes, with every element's shape tables spread over the component's
    // local node columns (zeros outside the element), so that the integration
    // sums the overlap of elements at shared nodes
    // (src/solver/compute_system_row_entries.hpp:83-97).
    std::vector<int> comp(d->num_beams > 0 ? d->num_beams : 0);
    for (int e = 0; e < d->num_beams; ++e) comp[e] = e;
    auto find = [&](int e) {
        while (comp[e] != e) e = comp[e] = comp[comp[e]];
        return e;
    };
    {
        std::vector<int> node_elem(nn, -1);
        for (int e = 0; e < d->num_beams; ++e) {
            const int n0 = d->beam_node_offsets[e], n1 = d->beam_node_offsets[e + 1];
            if (n1 - n0 < 2) return fail(err, KYN_ERR_INVALID, "beam needs >= 2 nodes, >= 1 qp, >= 1 section");
            for (int k = n0; k < n1; ++k) {
                const int id = d->beam_node_ids[k];
                if (id < 0 || id >= nn) return fail(err, KYN_ERR_INVALID, "beam node id out of range");
                for (int k2 = n0; k2 < k; ++k2)
                    if (d->beam_node_ids[k2] == id)
                        return fail(err, KYN_ERR_INVALID, "node listed twice in one beam element");
                if (node_elem[id] >= 0) {
                    const int a = find(node_elem[id]), b = find(e);
                    if (a != b) comp[std::max(a, b)] = std::min(a, b);
                } else {
                    node_elem[id] = e;
                }
            }
        }
    }
    // Condensed dense model: a multi-element beam larger than one FP64 system
    // (kMaxFP64SystemNodes), or a model that needs the dense bordered system
    // (below) but has more than kDenseModelMaxDofs unknowns.  Every element is
    // then its own component; the interior nodes of each are eliminated inside
    // the component (kyn_step_kernel.cuh, cond_component_terms).
    bool condense = false;
    if (d->num_beams > 0) {
        std::vector<int> group_nodes(d->num_beams, 0), group_elems(d->num_beams, 0);
        std::vector<int> seen(nn, -1);
        for (int e = 0; e < d->num_beams; ++e) {
            ++group_elems[find(e)];
            for (int k = d->beam_node_offsets[e]; k < d->beam_node_offsets[e + 1]; ++k) {
                const int id = d->beam_node_ids[k], r = find(e);
                if (seen[id] != r) {
                    seen[id] = r;
                    ++group_nodes[r];
                }
            }
        }
        for (int e = 0; e < d->num_beams; ++e)
            condense |= group_elems[e] > 1 && group_nodes[e] > kMaxFP64SystemNodes;
        if (!condense && needs_dense_beams(d) && dense_unknowns(d, true) > kDenseModelMaxDofs) condense = true;
        if (condense)
            for (int e = 0; e < d->num_beams; ++e) comp[e] = e;
    }
    std::vector<int> comp_index(d->num_beams > 0 ? d->num_beams : 0, -1);
    std::vector<std::vector<int>> comp_elems;
    for (int e = 0; e < d->num_beams; ++e) {
        const int r = find(e);
        if (comp_index[r] < 0) {
            comp_index[r] = static_cast<int>(comp_elems.size());
            comp_elems.emplace_back();
        }
        comp_elems[comp_index[r]].push_back(e);
    }
    if (comp_elems.size() > static_cast<size_t>(kMaxClusterBeams))
        return fail(err, KYN_ERR_UNSUPPORTED, "more than 8 beams in one model");
    M.num_elements = d->num_beams > 0 ? d->num_beams : 0;
    M.elem_row.assign(M.num_elements + 1, 0);
    for (int e = 0; e < M.num_elements; ++e)
        M.elem_row[e + 1] = M.elem_row[e] + d->beam_node_offsets[e + 1] - d->beam_node_offsets[e];
    M.beams.resize(comp_elems.size());

    std::vector<int> local_of(nn, -1);
    for (size_t ci = 0; ci < comp_elems.size(); ++ci) {
        HostBeam& B = M.beams[ci];
        // local nodes in order of first appearance, element by element (the
        // elements of a condensed model share nodes across components)
        int qtot = 0;
        for (int e : comp_elems[ci]) {
            const int n0 = d->beam_node_offsets[e], n1 = d->beam_node_offsets[e + 1];
            std::vector<int> loc;
            for (int k = n0; k < n1; ++k) {
                const int id = d->beam_node_ids[k];
                if (local_of[id] < 0) {
                    local_of[id] = static_cast<int>(B.node_ids.size());
                    B.node_ids.push_back(id);
                }
                M.node_beam[id] = static_cast<int>(ci);
                M.node_local[id] = local_of[id];
                loc.push_back(local_of[id]);
            }
            B.elem_ids.push_back(e);
            B.elem_local.push_back(loc);
            qtot += d->beam_qp_offsets[e + 1] - d->beam_qp_offsets[e];
        }
        for (int id : B.node_ids) local_of[id] = -1;
        B.N = static_cast<int>(B.node_ids.size());
        B.Q = qtot;
        if (B.N > 32 || B.Q > 64)
            return fail(err, KYN_ERR_UNSUPPORTED, "beam larger than 32 nodes or 64 qps");
        const int N = B.N, Q = B.Q;
        const SlabLayout L = make_slab_layout(N, Q);
        B.slab.assign(L.total, 0.);
        double* S = B.slab.data();
        int qo = 0;   // first quadrature point of the element in the component
        for (size_t ei = 0; ei < comp_elems[ci].size(); ++ei) {
            const int e = comp_elems[ci][ei];
            const std::vector<int>& loc = B.elem_local[ei];
            const int s0 = d->beam_section_offsets[e], s1 = d->beam_section_offsets[e + 1];
            const int q0 = d->beam_qp_offsets[e], q1 = d->beam_qp_offsets[e + 1];
            const int NE = static_cast<int>(loc.size()), QE = q1 - q0;
            if (QE < 1 || s1 - s0 < 1)
                return fail(err, KYN_ERR_INVALID, "beam needs >= 2 nodes, >= 1 qp, >= 1 section");
            for (int s = s0 + 1; s < s1; ++s)
                if (!(d->section_position[s] > d->section_position[s - 1]))
                    return fail(err, KYN_ERR_INVALID, "section positions must increase");
            std::vector<int> enode(NE);
            for (int k = 0; k < NE; ++k) enode[k] = B.node_ids[loc[k]];
            if (fill_element_qps(d, e, enode, loc, N, qo, L, S, err) != KYN_OK) return KYN_ERR_INVALID;
            qo += QE;
        }
        init_node_state(d, B, L, S);
    }
    if (lumped) {
        // one system over all nodes, no quadrature points
        M.beams.resize(1);
        HostBeam& B = M.beams[0];
        B.N = nn;
        B.Q = 0;
        B.lumped = true;
        for (int n = 0; n < nn; ++n) {
            B.node_ids.push_back(n);
            M.node_beam[n] = 0;
            M.node_local[n] = n;
        }
        const SlabLayout L = make_slab_layout(B.N, 0);
        B.slab.assign(L.total, 0.);
        init_node_state(d, B, L, B.slab.data());
    }

    // A model with beam elements whose constraints the per-beam systems cannot
    // take -- a joint whose base node is a beam node (beams coupled to each
    // other, or a beam carrying a position-only node), or three-row
    // constraints -- is solved as one dense bordered system (dense_kernel),
    // as the reference assembles it (src/solver/create_full_matrix.hpp).  Its
    // beam components keep their constant data (appended to the dense slab
    // below); every node joins the one system record.
    const bool dense_beams = !lumped && (condense || needs_dense_beams(d));
    std::vector<HostBeam> comps;
    if (dense_beams) {
        if (M.beams.size() > static_cast<size_t>(kMaxDenseComps))
            return fail(err, KYN_ERR_UNSUPPORTED, "more than 8 beams in a dense model");
        comps = std::move(M.beams);
        M.beams.assign(1, HostBeam{});
        HostBeam& B = M.beams[0];
        B.N = nn;
        B.Q = 0;
        for (int n = 0; n < nn; ++n) {
            B.node_ids.push_back(n);
            M.node_beam[n] = 0;
            M.node_local[n] = n;
        }
        for (int e = 0; e < d->num_beams; ++e) {
            B.elem_ids.push_back(e);
            B.elem_local.emplace_back(d->beam_node_ids + d->beam_node_offsets[e],
                                      d->beam_node_ids + d->beam_node_offsets[e + 1]);
        }
        const SlabLayout L = make_slab_layout(nn, 0);
        B.slab.assign(L.total, 0.);
        init_node_state(d, B, L, B.slab.data());
        B.n_comps = static_cast<int>(comps.size());
        for (const HostBeam& cb : comps) {
            B.comp_maxN = std::max(B.comp_maxN, cb.N);
            B.comp_maxQ = std::max(B.comp_maxQ, cb.Q);
        }
        if (condense) {
            // bordered-system unknowns: the nodes that are not interior to one
            // component, then the constraint rows
            std::vector<int> ncomp(nn, 0);
            for (const HostBeam& cb : comps)
                for (int id : cb.node_ids) ++ncomp[id];
            const std::vector<int> other = node_signatures(d, false);
            B.cond_nd = 0;
            for (int n = 0; n < nn; ++n)
                if (!(ncomp[n] == 1 && other[n] == 0)) B.cond_nd += 6;
            for (int c = 0; c < d->num_constraints; ++c) B.cond_nd += constraint_rows(d->constraint_type[c]);
            if (B.cond_nd > kCondMaxDofs)
                return fail(err, KYN_ERR_UNSUPPORTED, "condensed model with more than 160 bordered-system unknowns");
        }
    }

    // point masses and springs join the beam that holds their nodes
    // (src/elements/masses/create_masses.hpp, src/elements/springs/create_springs.hpp)
    std::vector<std::vector<double>> lrec_mass(M.beams.size()), lrec_spring(M.beams.size());
    std::vector<int> node_mass(nn, 0);
    for (int e = 0; e < n_mass; ++e) {
        const int node = d->mass_node[e];
        if (node < 0 || node >= nn) return fail(err, KYN_ERR_INVALID, "mass node out of range");
        const int b = M.node_beam[node];
        if (b < 0) return fail(err, KYN_ERR_UNSUPPORTED, "point mass on a node outside the beams");
        auto& r = lrec_mass[b];
        r.push_back(static_cast<double>(M.node_local[node]));
        r.insert(r.end(), d->mass_matrix + e * 36, d->mass_matrix + e * 36 + 36);
        r.insert(r.end(), d->node_x0 + node * 7 + 3, d->node_x0 + node * 7 + 7);
        node_mass[node] = 1;
    }
    M.spring_nodes.assign(n_spring * 2, 0);
    for (int e = 0; e < n_spring; ++e) {
        const int n1 = d->spring_nodes[2 * e], n2 = d->spring_nodes[2 * e + 1];
        if (n1 < 0 || n1 >= nn || n2 < 0 || n2 >= nn || n1 == n2)
            return fail(err, KYN_ERR_INVALID, "spring nodes out of range");
        const int b = M.node_beam[n1];
        if (b < 0 || M.node_beam[n2] != b)
            return fail(err, KYN_ERR_UNSUPPORTED, "spring between nodes of different beams");
        auto& r = lrec_spring[b];
        r.push_back(static_cast<double>(M.node_local[n1]));
        r.push_back(static_cast<double>(M.node_local[n2]));
        for (int c = 0; c < 3; ++c) r.push_back(d->node_x0[n2 * 7 + c] - d->node_x0[n1 * 7 + c]);
        r.push_back(d->spring_length[e]);
        r.push_back(d->spring_stiffness[e]);
        M.spring_nodes[2 * e] = n1;
        M.spring_nodes[2 * e + 1] = n2;
    }
    for (size_t b = 0; b < M.beams.size(); ++b) {
        HostBeam& B = M.beams[b];
        B.n_mass = static_cast<int>(lrec_mass[b].size()) / kMassRec;
        B.n_spring = static_cast<int>(lrec_spring[b].size()) / kSpringRec;
        if (B.n_mass > KYN_LUMPED_MAX_MASSES || B.n_spring > KYN_LUMPED_MAX_SPRINGS)
            return fail(err, KYN_ERR_UNSUPPORTED, "more point masses or springs than one system holds");
        B.lumped_off = static_cast<int>(B.slab.size());
        B.slab.insert(B.slab.end(), lrec_mass[b].begin(), lrec_mass[b].end());
        B.slab.insert(B.slab.end(), lrec_spring[b].begin(), lrec_spring[b].end());
    }
    if (dense_beams) {
        // [header: kCompHead doubles per component][component slabs], every
        // slab at an even double offset (its arrays are 16-byte aligned)
        HostBeam& B = M.beams[0];
        if (B.slab.size() & 1) B.slab.push_back(0.);
        B.comps_off = static_cast<int>(B.slab.size());
        std::vector<double> head(kCompHead * comps.size(), 0.);
        size_t at = (head.size() + 1) & ~static_cast<size_t>(1);
        std::vector<double> body;
        for (size_t ci = 0; ci < comps.size(); ++ci) {
            const HostBeam& cb = comps[ci];
            head[ci * kCompHead + 0] = static_cast<double>(at + body.size());
            head[ci * kCompHead + 1] = cb.N;
            head[ci * kCompHead + 2] = cb.Q;
            for (int k = 0; k < cb.N; ++k) head[ci * kCompHead + 3 + k] = cb.node_ids[k];
            body.insert(body.end(), cb.slab.begin(), cb.slab.end());
            if (body.size() & 1) body.push_back(0.);
        }
        if (B.cond_nd > 0)  // condensation workspaces [6Nc][6Nc + 1]
            for (size_t ci = 0; ci < comps.size(); ++ci) {
                const int mc = 6 * comps[ci].N;
                head[ci * kCompHead + kCompWork] = static_cast<double>(at + body.size());
                body.insert(body.end(), static_cast<size_t>(mc) * (mc + 1), 0.);
                if (body.size() & 1) body.push_back(0.);
            }
        head.resize(at, 0.);
        B.slab.insert(B.slab.end(), head.begin(), head.end());
        B.slab.insert(B.slab.end(), body.begin(), body.end());
    }
    // A node outside every beam element is allowed only as the hub of a rotor
    // (the base node of the joints, held by one single-node BC) or as a node
    // of a drive train: shaft base (held by one BC) -> revolute joint ->
    // azimuth [-> rigid joint -> hub], whose last node is the joints' base.
    const int ncon = (d->num_constraints > 0 && d->constraint_type) ? d->num_constraints : 0;
    auto base_of = [&](int c) { return d->constraint_base_node ? d->constraint_base_node[c] : -1; };
    // A lumped model with three-row constraints or joints between its nodes is
    // solved as the reference's dense bordered system (one CTA, pivoted LU);
    // a dense model takes its revolute joints as constraint rows, not as a
    // drive train.
    bool dense = dense_beams;
    for (int c = 0; c < ncon && lumped; ++c) {
        const int t = d->constraint_type[c];
        dense |= is_hub_joint(t) || t >= KYN_CONSTRAINT_FIXED_BC_3DOF || t == KYN_CONSTRAINT_REVOLUTE_JOINT;
    }
    for (int c = 0; c < ncon && !dense; ++c) {
        if (d->constraint_type[c] != KYN_CONSTRAINT_REVOLUTE_JOINT) continue;
        if (M.rev_con >= 0) return fail(err, KYN_ERR_UNSUPPORTED, "more than one revolute joint in a model");
        M.rev_con = c;
    }
    if (M.rev_con >= 0) {
        const int sb = base_of(M.rev_con), az = d->constraint_target_node[M.rev_con];
        if (sb < 0 || sb >= nn || az < 0 || az >= nn || sb == az)
            return fail(err, KYN_ERR_INVALID, "revolute joint nodes out of range");
        if (M.node_beam[sb] >= 0 || M.node_beam[az] >= 0)
            return fail(err, KYN_ERR_UNSUPPORTED, "a revolute joint must join two nodes outside the beams");
        M.chain = {sb, az};
        for (int c = 0; c < ncon; ++c) {
            const int t = d->constraint_target_node[c];
            if (d->constraint_type[c] == KYN_CONSTRAINT_RIGID_JOINT && base_of(c) == az && t >= 0 && t < nn &&
                M.node_beam[t] < 0) {
                if (M.ah_con >= 0) return fail(err, KYN_ERR_UNSUPPORTED, "drive train branches after the azimuth");
                M.ah_con = c;
            }
        }
        if (M.ah_con >= 0) M.chain.push_back(d->constraint_target_node[M.ah_con]);
        M.hub = sb;
        for (int n = 0; n < nn; ++n)
            if (M.node_beam[n] < 0 && std::find(M.chain.begin(), M.chain.end(), n) == M.chain.end())
                return fail(err, KYN_ERR_UNSUPPORTED, "node not attached to any beam element");
    } else {
        for (int n = 0; n < nn; ++n) {
            if (M.node_beam[n] >= 0) continue;
            bool is_hub = false;
            for (int c = 0; c < ncon; ++c)
                is_hub |= is_hub_joint(d->constraint_type[c]) && base_of(c) == n;
            if (!is_hub) return fail(err, KYN_ERR_UNSUPPORTED, "node not attached to any beam element");
            if (M.hub >= 0) return fail(err, KYN_ERR_UNSUPPORTED, "more than one hub node in a model");
            M.hub = n;
        }
        if (M.hub >= 0) M.chain = {M.hub};
    }
    const int jbase = M.chain.empty() ? -1 : M.chain.back();  // base node of the root joints

    // constraints (src/constraints/constraints.hpp:76-266)
    M.con_beam.assign(d->num_constraints, -1);
    M.con_slot.assign(d->num_constraints, -1);
    if (d->num_constraints > 0 && (!d->constraint_type || !d->constraint_target_node))
        return fail(err, KYN_ERR_INVALID, "constraints need type and target node");
    std::vector<int> node_con(nn, -1);
    std::vector<std::vector<int>> node_cols(nn);   // constraint row blocks coupled to a node
    static const double ident7[7] = {0., 0., 0., 1., 0., 0., 0.};
    int joints = 0;
    if (!lumped && !dense_beams)
        for (int c = 0; c < d->num_constraints; ++c)
            if (d->constraint_type[c] >= KYN_CONSTRAINT_FIXED_BC_3DOF)
                return fail(err, KYN_ERR_UNSUPPORTED,
                            "three-row constraints are supported in models without beam elements");
    if (dense) {
        HostBeam& B = M.beams[0];
        B.dense = true;
        if (d->num_constraints > kMaxBeamConstraints)
            return fail(err, KYN_ERR_UNSUPPORTED, "more than 16 constraints in a dense model");
        const SlabLayout L = make_slab_layout(B.N, 0);
        std::vector<double> frames(static_cast<size_t>(d->num_constraints) * 9, 0.);
        bool any_revolute = false;
        for (int c = 0; c < d->num_constraints; ++c) {
            const int t = d->constraint_type[c];
            const int node = d->constraint_target_node[c];
            if (node < 0 || node >= nn) return fail(err, KYN_ERR_INVALID, "constraint node out of range");
            const bool joint = is_hub_joint(t) || t == KYN_CONSTRAINT_RIGID_JOINT_6DOF_TO_3DOF ||
                               t == KYN_CONSTRAINT_REVOLUTE_JOINT;
            if (t < KYN_CONSTRAINT_FIXED_BC || t > KYN_CONSTRAINT_RIGID_JOINT_6DOF_TO_3DOF)
                return fail(err, KYN_ERR_UNSUPPORTED, "constraint type outside the dense-model path");
            const int base = joint ? base_of(c) : -1;
            if (joint && (base < 0 || base >= nn || base == node))
                return fail(err, KYN_ERR_INVALID, "joint base node out of range");
            const int slot = B.nc++;
            M.con_beam[c] = 0;
            M.con_slot[c] = slot;
            B.con_node[slot] = node;
            B.con_base[slot] = base;
            B.con_type[slot] = t;
            B.con_row[slot] = c;
            node_cols[node].push_back(c);
            if (joint) node_cols[base].push_back(c);
            const double* x0 = d->node_x0 + node * 7;
            const double* ax = d->constraint_axis ? d->constraint_axis + c * 3 : nullptr;
            const double* u = (d->constraint_initial_displacement &&
                               (t == KYN_CONSTRAINT_PRESCRIBED_BC || t == KYN_CONSTRAINT_PRESCRIBED_BC_3DOF))
                                  ? d->constraint_initial_displacement + c * 7 : ident7;
            for (int k = 0; k < 7; ++k) B.slab[L.con_input + slot * 7 + k] = u[k];
            for (int k = 0; k < 3; ++k) {  // X0 (src/constraints/constraints.hpp:224-233, 268-290)
                if (t == KYN_CONSTRAINT_FIXED_BC || t == KYN_CONSTRAINT_FIXED_BC_3DOF)
                    B.con_X0[slot][k] = x0[k] - (ax ? ax[k] : 0.);
                else if (joint)
                    B.con_X0[slot][k] = x0[k] - d->node_x0[base * 7 + k];
                else
                    B.con_X0[slot][k] = 0.;
            }
            if (t == KYN_CONSTRAINT_ROTATION_CONTROL) {
                const double nrm = ax ? std::sqrt(ax[0] * ax[0] + ax[1] * ax[1] + ax[2] * ax[2]) : 0.;
                if (!(nrm > 0.)) return fail(err, KYN_ERR_INVALID, "rotation control needs a nonzero axis");
                for (int k = 0; k < 3; ++k) B.con_axis[slot][k] = ax[k] / nrm;
            }
            if (t == KYN_CONSTRAINT_REVOLUTE_JOINT) {
                const int rc = revolute_frame(ax, B.con_X0[slot], frames.data() + slot * 9, err);
                if (rc != KYN_OK) return rc;
                any_revolute = true;
            }
        }
        if (any_revolute) {  // the joints' frames after the slab's other records
            if (B.slab.size() & 1) B.slab.push_back(0.);
            B.frames_off = static_cast<int>(B.slab.size());
            B.slab.insert(B.slab.end(), frames.begin(), frames.begin() + B.nc * 9);
        }
    }
    for (int c = 0; c < d->num_constraints && !dense; ++c) {
        const int t = d->constraint_type[c];
        if (t != KYN_CONSTRAINT_FIXED_BC && t != KYN_CONSTRAINT_PRESCRIBED_BC && !is_hub_joint(t) &&
            t != KYN_CONSTRAINT_REVOLUTE_JOINT)
            return fail(err, KYN_ERR_UNSUPPORTED,
                        "only FixedBC, PrescribedBC, RigidJoint, RevoluteJoint and RotationControl constraints");
        const int node = d->constraint_target_node[c];
        if (node < 0 || node >= nn) return fail(err, KYN_ERR_INVALID, "constraint node out of range");
        if (c == M.rev_con || c == M.ah_con) {  // joints inside the drive train
            if (t == KYN_CONSTRAINT_RIGID_JOINT || t == KYN_CONSTRAINT_REVOLUTE_JOINT) {
                node_cols[base_of(c)].push_back(c);
                node_cols[node].push_back(c);
                continue;
            }
        }
        if (is_hub_joint(t)) {
            const int base = base_of(c);
            if (base < 0 || base >= nn) return fail(err, KYN_ERR_INVALID, "joint base node out of range");
            if (base != jbase || M.node_beam[node] < 0)
                return fail(err, KYN_ERR_UNSUPPORTED,
                            "joints must join a hub node (in no beam) to a beam node");
            node_cols[base].push_back(c);
            ++joints;
        }
        if (M.chain.size() > 1 && node != M.hub &&
            std::find(M.chain.begin(), M.chain.end(), node) != M.chain.end())
            return fail(err, KYN_ERR_UNSUPPORTED, "a drive-train node other than the shaft base holds a BC");
        if (node == M.hub) {  // the hub's own boundary condition
            if (is_hub_joint(t) || M.hub_con >= 0)
                return fail(err, KYN_ERR_UNSUPPORTED, "the hub needs exactly one FixedBC or PrescribedBC");
            M.hub_con = c;
            M.hub_con_type = t;
            node_cols[node].push_back(c);
            continue;
        }
        if (node_con[node] >= 0)
            return fail(err, KYN_ERR_UNSUPPORTED, "two constraints on one node");
        node_con[node] = c;
        node_cols[node].push_back(c);
        const int e = M.node_beam[node];
        HostBeam& B = M.beams[e];
        if (B.nc >= kMaxBeamSystemConstraints)
            return fail(err, KYN_ERR_UNSUPPORTED, "more than 8 constraints on one beam");
        const int slot = B.nc++;
        M.con_beam[c] = e;
        M.con_slot[c] = slot;
        B.con_node[slot] = M.node_local[node];
        B.con_type[slot] = t;
        B.con_row[slot] = c;
        const SlabLayout L = make_slab_layout(B.N, B.Q);
        static const double ident[7] = {0., 0., 0., 1., 0., 0., 0.};
        if (t == KYN_CONSTRAINT_FIXED_BC) {
            const double* x0 = d->node_x0 + node * 7;
            for (int k = 0; k < 3; ++k)
                B.con_X0[slot][k] = x0[k] - (d->constraint_axis ? d->constraint_axis[c * 3 + k] : 0.);
            for (int k = 0; k < 7; ++k) B.slab[L.con_input + slot * 7 + k] = ident[k];
        } else if (is_hub_joint(t)) {
            // X0 = target x0 - base x0 (src/constraints/constraints.hpp:268-290)
            const double* x0 = d->node_x0 + node * 7;
            const double* xb = d->node_x0 + jbase * 7;
            for (int k = 0; k < 3; ++k) B.con_X0[slot][k] = x0[k] - xb[k];
            for (int k = 0; k < 7; ++k) B.slab[L.con_input + slot * 7 + k] = ident[k];
            if (t == KYN_CONSTRAINT_ROTATION_CONTROL) {
                // axes row 0 = UnitVector(axis) (src/constraints/constraints.hpp:321-328)
                const double* ax = d->constraint_axis ? d->constraint_axis + c * 3 : nullptr;
                const double nrm = ax ? std::sqrt(ax[0] * ax[0] + ax[1] * ax[1] + ax[2] * ax[2]) : 0.;
                if (!(nrm > 0.))
                    return fail(err, KYN_ERR_INVALID, "rotation control needs a nonzero axis");
                for (int k = 0; k < 3; ++k) B.con_axis[slot][k] = ax[k] / nrm;
            }
        } else {
            for (int k = 0; k < 3; ++k) B.con_X0[slot][k] = 0.;
            const double* u = d->constraint_initial_displacement
                                  ? d->constraint_initial_displacement + c * 7
                                  : ident;
            for (int k = 0; k < 7; ++k) B.slab[L.con_input + slot * 7 + k] = u[k];
        }
    }

    if (lumped && !dense)  // every node of a lumped model needs its 6 DOFs from a mass or a BC
        for (int n = 0; n < nn; ++n)
            if (!node_mass[n] && node_con[n] < 0)
                return fail(err, KYN_ERR_UNSUPPORTED,
                            "lumped-model node without a point mass or a boundary condition");
    if (M.hub >= 0 && (M.hub_con < 0 || joints == 0))
        return fail(err, KYN_ERR_UNSUPPORTED, "a hub node needs one BC and at least one joint");
    if (M.hub >= 0) {
        // every beam carries a copy of the hub's state
        const int h = M.hub;
        const double* x0 = d->node_x0 + h * 7;
        const double* u = d->node_u ? d->node_u + h * 7 : ident7;
        const int c = M.hub_con;
        for (auto& B : M.beams) {
            const SlabLayout L = make_slab_layout(B.N, B.Q);
            double* H = B.slab.data() + L.hub;
            for (int k = 0; k < 7; ++k) {
                H[hubrec::x0 + k] = x0[k];
                H[hubrec::q + k] = u[k];
                H[hubrec::q_prev + k] = u[k];
            }
            for (int k = 0; k < 3; ++k) H[hubrec::x + k] = x0[k] + u[k];
            qmul(u + 3, x0 + 3, H + hubrec::x + 3);
            for (int k = 0; k < 6; ++k) {
                H[hubrec::v + k] = d->node_v ? d->node_v[h * 6 + k] : 0.;
                H[hubrec::vd + k] = d->node_vd ? d->node_vd[h * 6 + k] : 0.;
                H[hubrec::a + k] = H[hubrec::vd + k];
            }
            for (int k = 0; k < 3; ++k) H[hubrec::tangent + k * 4] = 1.;
            const double* in = (M.hub_con_type == KYN_CONSTRAINT_PRESCRIBED_BC &&
                                d->constraint_initial_displacement)
                                   ? d->constraint_initial_displacement + c * 7 : ident7;
            for (int k = 0; k < 7; ++k) H[hubrec::input + k] = in[k];
            for (int k = 0; k < 3; ++k)
                H[hubrec::X0 + k] = (M.hub_con_type == KYN_CONSTRAINT_FIXED_BC)
                    ? x0[k] - (d->constraint_axis ? d->constraint_axis[c * 3 + k] : 0.) : 0.;
        }
    }
    // drive train: records 1 and 2 (state, the joint leading into the node)
    for (size_t r = 1; r < M.chain.size(); ++r) {
        const int n = M.chain[r], prev = M.chain[r - 1];
        const double* x0 = d->node_x0 + n * 7;
        const double* u = d->node_u ? d->node_u + n * 7 : ident7;
        double X0[3], axes[9] = {};
        for (int k = 0; k < 3; ++k) X0[k] = x0[k] - d->node_x0[prev * 7 + k];
        if (r == 1) {
            const int rc = revolute_frame(d->constraint_axis ? d->constraint_axis + M.rev_con * 3 : nullptr, X0,
                                          axes, err);
            if (rc != KYN_OK) return rc;
        }
        for (auto& B : M.beams) {
            const SlabLayout L = make_slab_layout(B.N, B.Q);
            double* H = B.slab.data() + L.hub + r * kHubDoubles;
            for (int k = 0; k < 7; ++k) {
                H[hubrec::x0 + k] = x0[k];
                H[hubrec::q + k] = u[k];
                H[hubrec::q_prev + k] = u[k];
                H[hubrec::input + k] = ident7[k];
            }
            for (int k = 0; k < 3; ++k) H[hubrec::x + k] = x0[k] + u[k];
            qmul(u + 3, x0 + 3, H + hubrec::x + 3);
            for (int k = 0; k < 6; ++k) {
                H[hubrec::v + k] = d->node_v ? d->node_v[n * 6 + k] : 0.;
                H[hubrec::vd + k] = d->node_vd ? d->node_vd[n * 6 + k] : 0.;
                H[hubrec::a + k] = H[hubrec::vd + k];
            }
            for (int k = 0; k < 3; ++k) H[hubrec::tangent + k * 4] = 1.;
            for (int k = 0; k < 3; ++k) H[hubrec::X0 + k] = X0[k];
            for (int k = 0; k < 9; ++k) H[hubrec::axes + k] = axes[k];
        }
    }

    // DOF map: exclusive scan of the nodes' DOFs in node-id order
    // (compute_node_freedom_map_table.hpp); constraint rows follow in order.
    // Every node carries 6 DOFs except, in a dense model, the position-only
    // nodes (FreedomSignature JustPosition: springs' nodes and targets of
    // three-row constraints, in no mass or six-DOF constraint).
    M.active.assign(nn, 6);
    if (dense) {
        std::vector<int> sig(nn, 0);
        for (int e = 0; e < n_mass; ++e) sig[d->mass_node[e]] |= kSigAll;
        for (int e = 0; e < n_spring; ++e) {
            sig[d->spring_nodes[2 * e]] |= kSigPosition;
            sig[d->spring_nodes[2 * e + 1]] |= kSigPosition;
        }
        for (int c = 0; c < d->num_constraints; ++c) {
            const int t = d->constraint_type[c];
            sig[d->constraint_target_node[c]] |= t >= KYN_CONSTRAINT_FIXED_BC_3DOF ? kSigPosition : kSigAll;
            if (is_hub_joint(t) || t == KYN_CONSTRAINT_RIGID_JOINT_6DOF_TO_3DOF || t == KYN_CONSTRAINT_REVOLUTE_JOINT)
                sig[base_of(c)] |= kSigAll;
        }
        for (int k = 0; dense_beams && k < d->beam_node_offsets[d->num_beams]; ++k)
            sig[d->beam_node_ids[k]] |= kSigAll;  // beam nodes (FreedomSignature AllComponents)
        for (int n = 0; n < nn; ++n) {
            if (sig[n] != kSigAll && sig[n] != kSigPosition)
                return fail(err, KYN_ERR_UNSUPPORTED, "dense-model node without six or three DOFs");
            M.active[n] = sig[n] == kSigAll ? 6 : 3;
        }
    }
    M.fmap.resize(nn);
    M.nsys = 0;
    for (int n = 0; n < nn; ++n) {
        M.fmap[n] = M.nsys;
        M.nsys += M.active[n];
    }
    M.con_rows.assign(d->num_constraints, 6);
    M.con_row_first.assign(d->num_constraints, 0);
    int crow = 0;
    for (int c = 0; c < d->num_constraints; ++c) {
        M.con_rows[c] = constraint_rows(d->constraint_type[c]);
        M.con_row_first[c] = crow;
        crow += M.con_rows[c];
    }
    M.ndofs = M.nsys + crow;
    if (dense && !condense && M.ndofs > kDenseModelMaxDofs)
        return fail(err, KYN_ERR_UNSUPPORTED, "dense model larger than 120 DOFs");

    // CRS graph: each row lists the DOFs it couples to, sorted ascending
    // (compute_row_ptrs.hpp, compute_col_inds.hpp, sort_crs_graph).
    M.row_ptrs.assign(M.ndofs + 1, 0);
    M.col_inds.clear();
    std::vector<int> cols;
    std::vector<int> row_node(M.nsys);
    for (int n = 0; n < nn; ++n)
        for (int c = 0; c < M.active[n]; ++c) row_node[M.fmap[n] + c] = n;
    for (int row = 0; row < M.ndofs; ++row) {
        cols.clear();
        if (row < M.nsys) {
            const int node = row_node[row];
            // own block first (compute_system_row_entries.hpp starts every row
            // with it), then the other nodes of every element holding the node
            for (int c = 0; c < M.active[node]; ++c) cols.push_back(M.fmap[node] + c);
            if (M.node_beam[node] >= 0 && !M.beams[M.node_beam[node]].lumped) {
                const HostBeam& B = M.beams[M.node_beam[node]];
                const int ln = M.node_local[node];
                for (const auto& loc : B.elem_local) {
                    if (std::find(loc.begin(), loc.end(), ln) == loc.end()) continue;
                    for (int k : loc)
                        if (k != ln)
                            for (int c = 0; c < 6; ++c) cols.push_back(M.fmap[B.node_ids[k]] + c);
                }
            }
            // a spring adds its other node's columns once per spring, also where
            // another element already added them (compute_system_col_inds.hpp:65-79)
            for (size_t e = 0; e + 1 < M.spring_nodes.size(); e += 2) {
                const int n1 = M.spring_nodes[e], n2 = M.spring_nodes[e + 1];
                if (n1 != node && n2 != node) continue;
                const int other = (n1 == node) ? n2 : n1;
                for (int c = 0; c < M.active[other]; ++c) cols.push_back(M.fmap[other] + c);
            }
            for (int con : node_cols[node])
                for (int c = 0; c < M.con_rows[con]; ++c) cols.push_back(M.nsys + M.con_row_first[con] + c);
        } else {
            int con = 0;
            while (con + 1 < d->num_constraints && M.con_row_first[con + 1] <= row - M.nsys) ++con;
            const int node = d->constraint_target_node[con];
            const int t = d->constraint_type[con];
            for (int c = 0; c < (t >= KYN_CONSTRAINT_FIXED_BC_3DOF ? 3 : 6); ++c) cols.push_back(M.fmap[node] + c);
            if (is_hub_joint(t) || t == KYN_CONSTRAINT_REVOLUTE_JOINT || t == KYN_CONSTRAINT_RIGID_JOINT_6DOF_TO_3DOF)
                for (int c = 0; c < 6; ++c) cols.push_back(M.fmap[d->constraint_base_node[con]] + c);
        }
        std::sort(cols.begin(), cols.end());
        M.col_inds.insert(M.col_inds.end(), cols.begin(), cols.end());
        M.row_ptrs[row + 1] = static_cast<int>(M.col_inds.size());
    }
    return KYN_OK;
}

}  // namespace kyn
