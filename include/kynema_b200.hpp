// kynema_b200.hpp -- C++ host shim that keeps Kynema's setup/step surface and
// calls the B200 beam path through the C ABI (kynema_b200.h).
//
// A caller of the reference writes
//     auto model = Model();  ... AddNode().SetElemLocation(s).SetPosition(...).Build();
//     model.AddBeamElement(ids, sections, quadrature);  model.AddFixedBC(ids[0]);
//     auto [state, elements, constraints, solver] = model.CreateSystemWithSolver<>();
//     Step(parameters, solver, elements, state, constraints);
// (src/model/model.hpp:74-693, src/step/step.hpp:42-124).  With this header the
// same code compiles against kynema_b200::, with a Context passed to
// CreateSystemWithSolver.  Errors of the library throw std::runtime_error;
// Step() returns false when the Newton loop reaches max_iter, as the reference.
#pragma once

#include <algorithm>
#include <array>
#include <cmath>
#include <memory>
#include <span>
#include <stdexcept>
#include <string>
#include <tuple>
#include <utility>
#include <vector>

#include "kynema_b200.h"

namespace kynema_b200 {

inline void check(kyn_ctx* ctx, int rc) {
    if (rc < 0) throw std::runtime_error(std::string("kynema_b200: ") + kyn_last_error(ctx));
}

// ---- math helpers used to build models (src/math/quaternion_operations.hpp) ----
inline std::array<double, 4> QuaternionCompose(const std::array<double, 4>& a,
                                               const std::array<double, 4>& b) {
    return {a[0] * b[0] - a[1] * b[1] - a[2] * b[2] - a[3] * b[3],
            a[0] * b[1] + a[1] * b[0] + a[2] * b[3] - a[3] * b[2],
            a[0] * b[2] - a[1] * b[3] + a[2] * b[0] + a[3] * b[1],
            a[0] * b[3] + a[1] * b[2] - a[2] * b[1] + a[3] * b[0]};
}

inline std::array<double, 3> RotateVectorByQuaternion(const std::array<double, 4>& q,
                                                      const std::array<double, 3>& v) {
    return {(q[0] * q[0] + q[1] * q[1] - q[2] * q[2] - q[3] * q[3]) * v[0] +
                2. * (q[1] * q[2] - q[0] * q[3]) * v[1] + 2. * (q[1] * q[3] + q[0] * q[2]) * v[2],
            2. * (q[1] * q[2] + q[0] * q[3]) * v[0] +
                (q[0] * q[0] - q[1] * q[1] + q[2] * q[2] - q[3] * q[3]) * v[1] +
                2. * (q[2] * q[3] - q[0] * q[1]) * v[2],
            2. * (q[1] * q[3] - q[0] * q[2]) * v[0] + 2. * (q[2] * q[3] + q[0] * q[1]) * v[1] +
                (q[0] * q[0] - q[1] * q[1] - q[2] * q[2] + q[3] * q[3]) * v[2]};
}

inline std::array<double, 4> RotationVectorToQuaternion(const std::array<double, 3>& phi) {
    const double angle = std::sqrt(phi[0] * phi[0] + phi[1] * phi[1] + phi[2] * phi[2]);
    if (std::abs(angle) < 1e-12) return {1., 0., 0., 0.};
    const double f = std::sin(angle / 2.) / angle;
    return {std::cos(angle / 2.), phi[0] * f, phi[1] * f, phi[2] * f};
}

// ---- device context ----------------------------------------------------------------
class Context {
public:
    explicit Context(int device = 0, size_t hbm_budget_bytes = 0)
        : ctx_(kyn_ctx_create(device, hbm_budget_bytes), &kyn_ctx_destroy) {
        if (!ctx_) throw std::runtime_error("kynema_b200: no CUDA device");
    }
    kyn_ctx* get() const { return ctx_.get(); }

private:
    std::shared_ptr<kyn_ctx> ctx_;
};

// ---- model description -------------------------------------------------------------
struct BeamSection {  // src/elements/beams/beam_section.hpp
    double position;
    std::array<std::array<double, 6>, 6> M_star;
    std::array<std::array<double, 6>, 6> C_star;
    BeamSection(double s, const std::array<std::array<double, 6>, 6>& m,
                const std::array<std::array<double, 6>, 6>& c)
        : position(s), M_star(m), C_star(c) {}
};

struct Node {  // src/model/node.hpp:35-60
    size_t id;
    std::array<double, 7> x0{0., 0., 0., 1., 0., 0., 0.};
    std::array<double, 7> u{0., 0., 0., 1., 0., 0., 0.};
    std::array<double, 6> v{};
    std::array<double, 6> vd{};
    double s = 0.;

    std::array<double, 7> DisplacedPosition() const {
        const auto q = QuaternionCompose({x0[3], x0[4], x0[5], x0[6]}, {u[3], u[4], u[5], u[6]});
        return {x0[0] + u[0], x0[1] + u[1], x0[2] + u[2], q[0], q[1], q[2], q[3]};
    }
    void Translate(const std::array<double, 3>& d) {
        for (int k = 0; k < 3; ++k) x0[k] += d[k];
    }
    void RotateAboutPoint(const std::array<double, 4>& q, const std::array<double, 3>& p) {
        const auto r = RotateVectorByQuaternion(q, {x0[0] - p[0], x0[1] - p[1], x0[2] - p[2]});
        for (int k = 0; k < 3; ++k) x0[k] = r[k] + p[k];
        const auto qn = QuaternionCompose(q, {x0[3], x0[4], x0[5], x0[6]});
        for (int k = 0; k < 4; ++k) x0[3 + k] = qn[k];
    }
    void SetVelocityAboutPoint(const std::array<double, 6>& vel, const std::array<double, 3>& p) {
        const auto dp = DisplacedPosition();
        const std::array<double, 3> r{dp[0] - p[0], dp[1] - p[1], dp[2] - p[2]};
        const std::array<double, 3> w{vel[3], vel[4], vel[5]};
        v = {vel[0] + (w[1] * r[2] - w[2] * r[1]), vel[1] + (w[2] * r[0] - w[0] * r[2]),
             vel[2] + (w[0] * r[1] - w[1] * r[0]), w[0], w[1], w[2]};
    }
    // src/model/node.hpp:233-262: rigid-body acceleration about a point
    void SetAccelerationAboutPoint(const std::array<double, 6>& acc, const std::array<double, 3>& omega,
                                   const std::array<double, 3>& p) {
        const auto dp = DisplacedPosition();
        const std::array<double, 3> r{dp[0] - p[0], dp[1] - p[1], dp[2] - p[2]};
        auto cross = [](const std::array<double, 3>& a, const std::array<double, 3>& b) {
            return std::array<double, 3>{a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2],
                                         a[0] * b[1] - a[1] * b[0]};
        };
        const auto ar = cross({acc[3], acc[4], acc[5]}, r);
        const auto wwr = cross(omega, cross(omega, r));
        vd = {acc[0] + ar[0] + wwr[0], acc[1] + ar[1] + wwr[1], acc[2] + ar[2] + wwr[2],
              acc[3], acc[4], acc[5]};
    }
};

class NodeBuilder {  // src/model/node.hpp:284-538
public:
    explicit NodeBuilder(Node& n) : node_(n) {}
    NodeBuilder& SetElemLocation(double s) { node_.s = s; return *this; }
    NodeBuilder& SetPosition(const std::array<double, 7>& p) { node_.x0 = p; return *this; }
    NodeBuilder& SetPosition(double x, double y, double z, double w, double i, double j, double k) {
        node_.x0 = {x, y, z, w, i, j, k};
        return *this;
    }
    NodeBuilder& SetPosition(double x, double y, double z) {
        node_.x0[0] = x; node_.x0[1] = y; node_.x0[2] = z;
        return *this;
    }
    NodeBuilder& SetDisplacement(const std::array<double, 7>& u) { node_.u = u; return *this; }
    NodeBuilder& SetVelocity(double x, double y, double z, double rx, double ry, double rz) {
        node_.v = {x, y, z, rx, ry, rz};
        return *this;
    }
    NodeBuilder& SetAcceleration(double x, double y, double z, double rx, double ry, double rz) {
        node_.vd = {x, y, z, rx, ry, rz};
        return *this;
    }
    size_t Build() const { return node_.id; }

private:
    Node& node_;
};

struct StepParameters {  // src/step/step_parameters.hpp:12-53
    bool is_dynamic_solve;
    size_t max_iter;
    double h, rho_inf, absolute_convergence_tol, relative_convergence_tol;
    int precision = KYN_PRECISION_FP64;
    int refine_iters = 0;
    StepParameters(bool dyn, size_t max_it, double h_, double rho, double a_tol = 1e-5,
                   double r_tol = 1e-3)
        : is_dynamic_solve(dyn), max_iter(max_it), h(h_), rho_inf(rho),
          absolute_convergence_tol(a_tol), relative_convergence_tol(r_tol) {}
    kyn_step_params c() const {
        return {is_dynamic_solve ? 1 : 0, static_cast<int32_t>(max_iter), h, rho_inf,
                absolute_convergence_tol, relative_convergence_tol, precision, refine_iters};
    }
};

// Device-resident model created from a Model; the four handles the reference's
// CreateSystemWithSolver returns all refer to it.
struct DeviceModel {
    explicit DeviceModel(const Context& c) : ctx(c) {}
    DeviceModel(const DeviceModel&) = delete;
    DeviceModel& operator=(const DeviceModel&) = delete;
    Context ctx;
    int id = -1;
    kyn_model_info info{};
    std::vector<double> node_fx;   // Beams::node_FX host mirror [element nodes][6]
    std::vector<size_t> elem_offset;
    bool fx_dirty = false;
    std::vector<double> errs;
    std::vector<std::pair<int, double*>> controls;  // RotationControl: constraint, signal
    ~DeviceModel() {
        if (id >= 0) kyn_model_destroy(ctx.get(), id);
    }
};

class State {  // src/state/state.hpp reads
public:
    explicit State(std::shared_ptr<DeviceModel> m) : m_(std::move(m)) {}
    std::vector<double> Get(int field) const {
        const size_t rows = field == KYN_FIELD_LAMBDA ? m_->info.num_constraints : m_->info.num_nodes;
        const size_t w = field == KYN_FIELD_TANGENT ? 36
                         : (field == KYN_FIELD_X0 || field == KYN_FIELD_X || field == KYN_FIELD_Q ||
                            field == KYN_FIELD_Q_PREV) ? 7 : 6;
        std::vector<double> out(rows * w);
        check(m_->ctx.get(), kyn_get_state(m_->ctx.get(), m_->id, field, out.data()));
        return out;
    }
    std::vector<double> q() const { return Get(KYN_FIELD_Q); }
    std::vector<double> v() const { return Get(KYN_FIELD_V); }
    std::vector<double> vd() const { return Get(KYN_FIELD_VD); }
    void SetExternalForces(const std::vector<double>& f) {  // State::f [nodes][6]
        check(m_->ctx.get(), kyn_model_set_loads(m_->ctx.get(), m_->id, KYN_LOAD_STATE_F, f.data()));
    }

private:
    std::shared_ptr<DeviceModel> m_;
};

class Elements {  // Beams::node_FX writes
public:
    explicit Elements(std::shared_ptr<DeviceModel> m) : m_(std::move(m)) {}
    // node_FX(element, node, component) = value
    void SetNodeFX(size_t element, size_t node, size_t component, double value) {
        m_->node_fx[(m_->elem_offset[element] + node) * 6 + component] = value;
        m_->fx_dirty = true;
    }

private:
    std::shared_ptr<DeviceModel> m_;
};

class Constraints {  // src/constraints/constraints.hpp:338-343
public:
    explicit Constraints(std::shared_ptr<DeviceModel> m) : m_(std::move(m)) {}
    void UpdateDisplacement(size_t id, const std::array<double, 7>& u) const {
        check(m_->ctx.get(), kyn_model_set_prescribed(m_->ctx.get(), m_->id, static_cast<int>(id), u.data()));
    }
    std::vector<double> lambda() const {
        std::vector<double> out(m_->info.num_constraints * 6);
        check(m_->ctx.get(), kyn_get_state(m_->ctx.get(), m_->id, KYN_FIELD_LAMBDA, out.data()));
        return out;
    }
    // Constraints::output, [constraints][3]: a revolute joint's rotation, angular
    // velocity and angular acceleration about its axis
    // (src/constraints/calculate_revolute_joint_output.hpp)
    std::vector<double> output() const {
        std::vector<double> out(m_->info.num_constraints * 3);
        check(m_->ctx.get(), kyn_get_state(m_->ctx.get(), m_->id, KYN_FIELD_CONSTRAINT_OUTPUT, out.data()));
        return out;
    }

private:
    std::shared_ptr<DeviceModel> m_;
};

class Solver {  // solver.convergence_err
public:
    explicit Solver(std::shared_ptr<DeviceModel> m) : m_(std::move(m)) {}
    const std::vector<double>& convergence_err() const { return m_->errs; }
    std::shared_ptr<DeviceModel> model() const { return m_; }

private:
    std::shared_ptr<DeviceModel> m_;
};

class Model {  // src/model/model.hpp:74-693
public:
    static constexpr size_t InvalidNodeID = 0;
    Model() = default;
    explicit Model(std::array<double, 3> g) : gravity_(g) {}
    void SetGravity(double x, double y, double z) { gravity_ = {x, y, z}; }

    NodeBuilder AddNode() {
        nodes_.push_back(Node{nodes_.size()});
        return NodeBuilder(nodes_.back());
    }
    Node& GetNode(size_t id) { return nodes_[id]; }

    size_t AddBeamElement(std::span<const size_t> node_ids, std::span<const BeamSection> sections,
                          std::span<const std::array<double, 2>> quadrature) {
        beams_.push_back({std::vector<size_t>(node_ids.begin(), node_ids.end()),
                          std::vector<BeamSection>(sections.begin(), sections.end()),
                          std::vector<std::array<double, 2>>(quadrature.begin(), quadrature.end())});
        return beams_.size() - 1;
    }
    void TranslateBeam(size_t e, const std::array<double, 3>& d) {
        for (auto n : beams_[e].nodes) nodes_[n].Translate(d);
    }
    void RotateBeamAboutPoint(size_t e, const std::array<double, 4>& q, const std::array<double, 3>& p) {
        for (auto n : beams_[e].nodes) nodes_[n].RotateAboutPoint(q, p);
    }
    void SetBeamVelocityAboutPoint(size_t e, const std::array<double, 6>& v, const std::array<double, 3>& p) {
        for (auto n : beams_[e].nodes) nodes_[n].SetVelocityAboutPoint(v, p);
    }
    void SetBeamAccelerationAboutPoint(size_t e, const std::array<double, 6>& a,
                                       const std::array<double, 3>& omega, const std::array<double, 3>& p) {
        for (auto n : beams_[e].nodes) nodes_[n].SetAccelerationAboutPoint(a, omega, p);
    }
    // src/model/model.hpp:305-311 AddMassElement: 6x6 mass (material frame) at a node
    size_t AddMassElement(size_t node, const std::array<std::array<double, 6>, 6>& mass) {
        masses_.push_back({node, mass});
        return masses_.size() - 1;
    }
    // src/model/model.hpp:376-389 AddSpringElement
    size_t AddSpringElement(size_t node1, size_t node2, double stiffness, double undeformed_length) {
        springs_.push_back({node1, node2, stiffness, undeformed_length});
        return springs_.size() - 1;
    }
    size_t AddFixedBC(size_t node) {
        cons_.push_back({KYN_CONSTRAINT_FIXED_BC, node, {0., 0., 0., 1., 0., 0., 0.}});
        return cons_.size() - 1;
    }
    size_t AddPrescribedBC(size_t node, const std::array<double, 7>& u0 = {0., 0., 0., 1., 0., 0., 0.}) {
        cons_.push_back({KYN_CONSTRAINT_PRESCRIBED_BC, node, u0});
        return cons_.size() - 1;
    }
    // three-row constraints on position-only nodes (src/model/model.hpp:570-611);
    // models without beam elements that use them run as their dense system
    size_t AddFixedBC3DOFs(size_t node) {
        cons_.push_back({KYN_CONSTRAINT_FIXED_BC_3DOF, node, {0., 0., 0., 1., 0., 0., 0.}});
        return cons_.size() - 1;
    }
    size_t AddPrescribedBC3DOFs(size_t node, const std::array<double, 7>& u0 = {0., 0., 0., 1., 0., 0., 0.}) {
        cons_.push_back({KYN_CONSTRAINT_PRESCRIBED_BC_3DOF, node, u0});
        return cons_.size() - 1;
    }
    size_t AddRigidJoint6DOFsTo3DOFs(const std::array<size_t, 2>& nodes) {
        cons_.push_back({KYN_CONSTRAINT_RIGID_JOINT_6DOF_TO_3DOF, nodes[1], {0., 0., 0., 1., 0., 0., 0.}, nodes[0]});
        return cons_.size() - 1;
    }
    // {base (hub), target} (src/model/model.hpp AddRigidJointConstraint)
    size_t AddRigidJointConstraint(const std::array<size_t, 2>& nodes) {
        cons_.push_back({KYN_CONSTRAINT_RIGID_JOINT, nodes[1], {0., 0., 0., 1., 0., 0., 0.}, nodes[0]});
        return cons_.size() - 1;
    }

    // {base (shaft base), target (azimuth or hub)}, joint axis (zero: the
    // base-to-target direction) and the torque read before every Step
    // (src/model/model.hpp:529-541 AddRevoluteJointConstraint)
    size_t AddRevoluteJointConstraint(const std::array<size_t, 2>& nodes,
                                      const std::array<double, 3>& axis, double* torque) {
        cons_.push_back({KYN_CONSTRAINT_REVOLUTE_JOINT, nodes[1], {0., 0., 0., 1., 0., 0., 0.},
                         nodes[0], axis, torque});
        return cons_.size() - 1;
    }
    // {base (hub), target}, rotation axis and the control signal read before
    // every Step (src/model/model.hpp:550-562 AddRotationControl)
    size_t AddRotationControl(const std::array<size_t, 2>& nodes, const std::array<double, 3>& axis,
                              double* control) {
        cons_.push_back({KYN_CONSTRAINT_ROTATION_CONTROL, nodes[1], {0., 0., 0., 1., 0., 0., 0.},
                         nodes[0], axis, control});
        return cons_.size() - 1;
    }

    std::tuple<State, Elements, Constraints, Solver> CreateSystemWithSolver(const Context& ctx) const {
        auto m = std::make_shared<DeviceModel>(ctx);
        WithDescription([&](const kyn_model_desc& d) {
            const int id = kyn_model_create(ctx.get(), &d);
            check(ctx.get(), id);
            m->id = id;
        });
        check(ctx.get(), kyn_model_info_get(ctx.get(), m->id, &m->info));
        size_t elem_nodes = 0;
        for (const auto& b : beams_) {
            m->elem_offset.push_back(elem_nodes);
            elem_nodes += b.nodes.size();
        }
        for (size_t k = 0; k < cons_.size(); ++k)
            if (cons_[k].control) m->controls.emplace_back(static_cast<int>(k), cons_[k].control);
        m->node_fx.assign(elem_nodes * 6, 0.);
        return {State(m), Elements(m), Constraints(m), Solver(m)};
    }

    // Calls f with the plain-array description of this model (kyn_model_desc,
    // valid during the call), the input of kyn_model_create.
    template <typename F>
    void WithDescription(F&& f) const {
        std::vector<double> x0, u, v, vd, s, spos, smass, sstiff, qxi, qw, cinit, caxis;
        std::vector<int32_t> bno{0}, bni, bso{0}, bqo{0}, ctype, cbase, ctarget;
        for (const auto& n : nodes_) {
            x0.insert(x0.end(), n.x0.begin(), n.x0.end());
            u.insert(u.end(), n.u.begin(), n.u.end());
            v.insert(v.end(), n.v.begin(), n.v.end());
            vd.insert(vd.end(), n.vd.begin(), n.vd.end());
            s.push_back(n.s);
        }
        for (const auto& b : beams_) {
            for (auto n : b.nodes) bni.push_back(static_cast<int32_t>(n));
            bno.push_back(static_cast<int32_t>(bni.size()));
            for (const auto& sec : b.sections) {
                spos.push_back(sec.position);
                for (const auto& row : sec.M_star) smass.insert(smass.end(), row.begin(), row.end());
                for (const auto& row : sec.C_star) sstiff.insert(sstiff.end(), row.begin(), row.end());
            }
            bso.push_back(static_cast<int32_t>(spos.size()));
            for (const auto& q : b.quad) {
                qxi.push_back(q[0]);
                qw.push_back(q[1]);
            }
            bqo.push_back(static_cast<int32_t>(qxi.size()));
        }
        for (const auto& c : cons_) {
            ctype.push_back(c.type);
            cbase.push_back(static_cast<int32_t>(c.base));
            ctarget.push_back(static_cast<int32_t>(c.node));
            cinit.insert(cinit.end(), c.u0.begin(), c.u0.end());
            caxis.insert(caxis.end(), c.axis.begin(), c.axis.end());
        }
        kyn_model_desc d{};
        d.num_nodes = static_cast<int32_t>(nodes_.size());
        d.node_x0 = x0.data(); d.node_u = u.data(); d.node_v = v.data(); d.node_vd = vd.data();
        d.node_s = s.data();
        d.num_beams = static_cast<int32_t>(beams_.size());
        d.beam_node_offsets = bno.data(); d.beam_node_ids = bni.data();
        d.beam_section_offsets = bso.data(); d.section_position = spos.data();
        d.section_mass = smass.data(); d.section_stiffness = sstiff.data();
        d.beam_qp_offsets = bqo.data(); d.qp_xi = qxi.data(); d.qp_weight = qw.data();
        d.num_constraints = static_cast<int32_t>(cons_.size());
        d.constraint_type = ctype.data(); d.constraint_base_node = cbase.data();
        d.constraint_target_node = ctarget.data(); d.constraint_axis = caxis.data();
        d.constraint_initial_displacement = cinit.data();
        for (int k = 0; k < 3; ++k) d.gravity[k] = gravity_[k];
        std::vector<int32_t> mnode, snodes;
        std::vector<double> mmat, sk, sl;
        for (const auto& ms : masses_) {
            mnode.push_back(static_cast<int32_t>(ms.node));
            for (const auto& row : ms.mass) mmat.insert(mmat.end(), row.begin(), row.end());
        }
        for (const auto& sp : springs_) {
            snodes.push_back(static_cast<int32_t>(sp.n1));
            snodes.push_back(static_cast<int32_t>(sp.n2));
            sk.push_back(sp.k);
            sl.push_back(sp.l0);
        }
        d.num_masses = static_cast<int32_t>(masses_.size());
        d.mass_node = mnode.data(); d.mass_matrix = mmat.data();
        d.num_springs = static_cast<int32_t>(springs_.size());
        d.spring_nodes = snodes.data(); d.spring_stiffness = sk.data(); d.spring_length = sl.data();
        f(static_cast<const kyn_model_desc&>(d));
    }

private:
    struct Beam {
        std::vector<size_t> nodes;
        std::vector<BeamSection> sections;
        std::vector<std::array<double, 2>> quad;
    };
    struct Con {
        int type;
        size_t node;
        std::array<double, 7> u0;
        size_t base = 0;
        std::array<double, 3> axis{0., 0., 0.};
        double* control = nullptr;
    };
    struct Mass {
        size_t node;
        std::array<std::array<double, 6>, 6> mass;
    };
    struct Spring {
        size_t n1, n2;
        double k, l0;
    };
    std::vector<Mass> masses_;
    std::vector<Spring> springs_;
    std::array<double, 3> gravity_{0., 0., 0.};
    std::vector<Node> nodes_;
    std::vector<Beam> beams_;
    std::vector<Con> cons_;
};

// kynema::Step (src/step/step.hpp:42-124): true when the Newton loop converged.
inline bool Step(const StepParameters& parameters, Solver& solver, Elements&, State&, Constraints&) {
    auto m = solver.model();
    kyn_ctx* c = m->ctx.get();
    if (m->fx_dirty) {
        check(c, kyn_model_set_loads(c, m->id, KYN_LOAD_NODE_FX, m->node_fx.data()));
        m->fx_dirty = false;
    }
    // control signals into the constraints' input slot 0
    // (src/constraints/constraints.hpp:345-352 UpdateViews)
    for (const auto& [cid, signal] : m->controls) {
        const double u[7] = {*signal, 0., 0., 1., 0., 0., 0.};
        check(c, kyn_model_set_prescribed(c, m->id, cid, u));
    }
    const kyn_step_params p = parameters.c();
    int status = 0, iters = 0;
    check(c, kyn_step(c, &m->id, 1, &p, &status, &iters));
    m->errs.assign(static_cast<size_t>(std::max(iters, p.max_iter)), 0.);
    int n = 0;
    check(c, kyn_get_convergence(c, m->id, m->errs.data(), &n));
    m->errs.resize(static_cast<size_t>(n));
    if (status < 0)
        throw std::runtime_error("kynema_b200: step failed with status " + std::to_string(status));
    return status == KYN_OK;
}

}  // namespace kynema_b200
