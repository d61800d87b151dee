// kynema_b200_interfaces.hpp -- the blade interface of Kynema on the B200 path.
//
// A code that couples a wind-turbine blade to an aerodynamics or CFD solver
// uses the reference's BladeInterface (src/interfaces/blade/blade_interface.hpp):
// it describes the blade by a reference axis, twist and 6x6 sections
// (BladeInterfaceBuilder / components::BeamBuilder), writes nodal loads into
// Blade().nodes[i].loads, calls Step(), and reads the nodes' position,
// displacement, velocity and acceleration back.  This header keeps that
// surface; the blade becomes one beam element of the requested order built
// through the C++ shim (kynema_b200.hpp), and each Step() is one kyn_step of
// the device model.  NetCDF and YAML output of the reference are not part of
// this path; SetOutputFile only records the path.
#pragma once

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <limits>
#include <memory>
#include <numbers>
#include <stdexcept>
#include <string>
#include <vector>

#include "kynema_b200.hpp"

namespace kynema_b200::interfaces {

// ---- geometry helpers (src/math/interpolation.hpp, least_squares_fit.hpp,
//      project_points_to_target_polynomial.hpp, quaternion_operations.hpp,
//      matrix_operations.hpp) ----------------------------------------------------------
namespace math {

using M3 = std::array<std::array<double, 3>, 3>;
using M6 = std::array<std::array<double, 6>, 6>;

// P_n(x) by the three-term recurrence
inline double Legendre(size_t n, double x) {
    if (n == 0) return 1.;
    double p2 = 1., p1 = x, p = x;
    for (size_t i = 2; i <= n; ++i) {
        const double di = static_cast<double>(i);
        p = ((2. * di - 1.) * x * p1 - (di - 1.) * p2) / di;
        p2 = p1;
        p1 = p;
    }
    return p;
}

// Gauss-Lobatto-Legendre points of a polynomial order, ascending: the end
// points and the roots of (1 - x^2) P'_order, found by Newton's method from the
// Chebyshev-Lobatto points (interpolation.hpp:169-230).
inline std::vector<double> GenerateGLLPoints(size_t order) {
    if (order < 1) throw std::invalid_argument("polynomial order must be >= 1");
    const size_t n = order + 1;
    std::vector<double> x(n, 0.);
    x.front() = -1.;
    x.back() = 1.;
    for (size_t i = 1; i < order; ++i) {
        double xi = -std::cos(static_cast<double>(i) * std::numbers::pi / static_cast<double>(order));
        bool done = false;
        for (int it = 0; it < 1000 && !done; ++it) {
            const double old = xi;
            const double pn = Legendre(n - 1, xi), pm = Legendre(n - 2, xi);
            xi -= (xi * pn - pm) / (static_cast<double>(n) * pn);
            done = std::abs(xi - old) <= std::numeric_limits<double>::epsilon();
        }
        if (!done) throw std::runtime_error("GLL point iteration did not converge");
        x[i] = xi;
    }
    return x;
}

inline std::vector<double> LagrangeWeights(double x, const std::vector<double>& xs) {
    std::vector<double> w(xs.size(), 1.);
    for (size_t j = 0; j < xs.size(); ++j)
        for (size_t m = 0; m < xs.size(); ++m)
            if (m != j) w[j] *= (x - xs[m]) / (xs[j] - xs[m]);
    return w;
}

inline std::vector<double> LagrangeDerivWeights(double x, const std::vector<double>& xs) {
    std::vector<double> w(xs.size(), 0.);
    for (size_t j = 0; j < xs.size(); ++j)
        for (size_t i = 0; i < xs.size(); ++i) {
            if (i == j) continue;
            double p = 1. / (xs[j] - xs[i]);
            for (size_t m = 0; m < xs.size(); ++m)
                if (m != i && m != j) p *= (x - xs[m]) / (xs[j] - xs[m]);
            w[j] += p;
        }
    return w;
}

// Linear interpolation on a sorted grid, clamped at its ends.
inline double LinearInterp(double x, const std::vector<double>& xs, const std::vector<double>& v) {
    if (xs.empty()) return 0.;
    if (x <= xs.front()) return v.front();
    if (x >= xs.back()) return v.back();
    const size_t k = static_cast<size_t>(std::lower_bound(xs.begin(), xs.end(), x) - xs.begin());
    const double u = (x - xs[k - 1]) / (xs[k] - xs[k - 1]);
    return (1. - u) * v[k - 1] + u * v[k];
}

inline M3 QuaternionToRotationMatrix(const std::array<double, 4>& q) {
    const double w = q[0], x = q[1], y = q[2], z = q[3];
    return {{{w * w + x * x - y * y - z * z, 2. * (x * y - w * z), 2. * (x * z + w * y)},
             {2. * (x * y + w * z), w * w - x * x + y * y - z * z, 2. * (y * z - w * x)},
             {2. * (x * z - w * y), 2. * (y * z + w * x), w * w - x * x - y * y + z * z}}};
}

// The quaternion of a rotation matrix, from its largest diagonal combination
// (quaternion_operations.hpp:63-120).
inline std::array<double, 4> RotationMatrixToQuaternion(const M3& m) {
    const double a = m[1][1] + m[2][2], b = m[1][1] - m[2][2];
    const std::array<double, 4> vals{m[0][0] + a, m[0][0] - a, -m[0][0] + b, -m[0][0] - b};
    const size_t k = static_cast<size_t>(std::max_element(vals.begin(), vals.end()) - vals.begin());
    const double t = std::sqrt(vals[k] + 1.), c = 0.5 / t;
    switch (k) {
        case 0: return {0.5 * t, (m[2][1] - m[1][2]) * c, (m[0][2] - m[2][0]) * c, (m[1][0] - m[0][1]) * c};
        case 1: return {(m[2][1] - m[1][2]) * c, 0.5 * t, (m[0][1] + m[1][0]) * c, (m[0][2] + m[2][0]) * c};
        case 2: return {(m[0][2] - m[2][0]) * c, (m[0][1] + m[1][0]) * c, 0.5 * t, (m[1][2] + m[2][1]) * c};
        default: return {(m[1][0] - m[0][1]) * c, (m[0][2] + m[2][0]) * c, (m[1][2] + m[2][1]) * c, 0.5 * t};
    }
}

inline std::array<double, 3> Unit(const std::array<double, 3>& v) {
    const double n = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    return {v[0] / n, v[1] / n, v[2] / n};
}

// Orientation whose first axis is the tangent, turned by twist (degrees) about
// it; the second axis lies in the plane of the tangent and y (or x when the
// tangent is near y) (quaternion_operations.hpp:334-362).
inline std::array<double, 4> TangentTwistToQuaternion(const std::array<double, 3>& tangent, double twist) {
    const auto e1 = Unit(tangent);
    std::array<double, 3> t{0., 1., 0.};
    if (std::abs(e1[0] * t[0] + e1[1] * t[1] + e1[2] * t[2]) > 0.9) t = {1., 0., 0.};
    const double a = e1[0] * t[0] + e1[1] * t[1] + e1[2] * t[2];
    const auto e2 = Unit({t[0] - e1[0] * a, t[1] - e1[1] * a, t[2] - e1[2] * a});
    const std::array<double, 3> e3{e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2],
                                   e1[0] * e2[1] - e1[1] * e2[0]};
    const auto q_tan = RotationMatrixToQuaternion({{{e1[0], e2[0], e3[0]},
                                                    {e1[1], e2[1], e3[1]},
                                                    {e1[2], e2[2], e3[2]}}});
    const double tw = twist * std::numbers::pi / 180.;
    const auto q_twist = RotationVectorToQuaternion({e1[0] * tw, e1[1] * tw, e1[2] * tw});
    return QuaternionCompose(q_twist, q_tan);
}

// diag(R, R) m diag(R, R)^T
inline M6 RotateMatrix6(const M6& m, const std::array<double, 4>& q) {
    const auto R = QuaternionToRotationMatrix(q);
    auto r = [&](size_t i, size_t k) {
        return (i / 3 == k / 3) ? R[i % 3][k % 3] : 0.;
    };
    M6 t{}, o{};
    for (size_t i = 0; i < 6; ++i)
        for (size_t j = 0; j < 6; ++j)
            for (size_t k = 0; k < 6; ++k) t[i][j] += r(i, k) * m[k][j];
    for (size_t i = 0; i < 6; ++i)
        for (size_t j = 0; j < 6; ++j)
            for (size_t k = 0; k < 6; ++k) o[i][j] += t[i][k] * r(j, k);
    return o;
}

// Trapezoidal rule on a grid mapped to [-1, 1] (src/elements/beams/beam_quadrature.hpp:11-28).
inline std::vector<std::array<double, 2>> CreateTrapezoidalQuadrature(const std::vector<double>& grid) {
    const size_t n = grid.size();
    const auto [lo, hi] = std::minmax_element(grid.begin(), grid.end());
    const double g0 = *lo, range = *hi - *lo;
    std::vector<std::array<double, 2>> q{{-1., (grid[1] - grid[0]) / range}};
    for (size_t i = 1; i + 1 < n; ++i)
        q.push_back({2. * (grid[i] - g0) / range - 1., (grid[i + 1] - grid[i - 1]) / range});
    q.push_back({1., (grid[n - 1] - grid[n - 2]) / range});
    return q;
}

// Node coordinates of a polynomial through key points: least squares with the
// first and last node held at the first and last key point (interior rows are
// the normal equations), solved by Gaussian elimination with partial pivoting
// (least_squares_fit.hpp: MapGeometricLocations, ComputeShapeFunctionValues,
// PerformLeastSquaresFitting).
inline std::vector<std::array<double, 3>> FitNodes(const std::vector<double>& node_xi,
                                                   const std::vector<double>& kp_grid,
                                                   const std::vector<std::array<double, 3>>& kp) {
    const size_t p = node_xi.size(), n = kp.size();
    const double g0 = kp_grid.front(), span = kp_grid.back() - kp_grid.front();
    if (span == 0.) throw std::invalid_argument("reference axis grid has zero length");
    std::vector<std::vector<double>> phi(p, std::vector<double>(n));   // phi[node][key point]
    for (size_t k = 0; k < n; ++k) {
        const auto w = LagrangeWeights(2. * (kp_grid[k] - g0) / span - 1., node_xi);
        for (size_t i = 0; i < p; ++i) phi[i][k] = w[i];
    }
    std::vector<std::vector<double>> A(p, std::vector<double>(p, 0.));
    std::vector<std::array<double, 3>> B(p, {0., 0., 0.});
    A[0][0] = 1.;
    A[p - 1][p - 1] = 1.;
    B[0] = kp.front();
    B[p - 1] = kp.back();
    for (size_t i = 1; i + 1 < p; ++i) {
        for (size_t j = 0; j < p; ++j) {
            double s = 0.;
            for (size_t k = 0; k < n; ++k) s += phi[i][k] * phi[j][k];
            A[i][j] = s;
        }
        for (size_t k = 0; k < n; ++k)
            for (int d = 0; d < 3; ++d) B[i][d] += phi[i][k] * kp[k][d];
    }
    for (size_t c = 0; c < p; ++c) {
        size_t piv = c;
        for (size_t r = c + 1; r < p; ++r)
            if (std::abs(A[r][c]) > std::abs(A[piv][c])) piv = r;
        std::swap(A[c], A[piv]);
        std::swap(B[c], B[piv]);
        for (size_t r = c + 1; r < p; ++r) {
            const double l = A[r][c] / A[c][c];
            for (size_t j = c; j < p; ++j) A[r][j] -= l * A[c][j];
            for (int d = 0; d < 3; ++d) B[r][d] -= l * B[c][d];
        }
    }
    std::vector<std::array<double, 3>> X(p);
    for (size_t r = p; r-- > 0;) {
        for (int d = 0; d < 3; ++d) {
            double s = B[r][d];
            for (size_t j = r + 1; j < p; ++j) s -= A[r][j] * X[j][d];
            X[r][d] = s / A[r][r];
        }
    }
    return X;
}

// Values of the order (m-1) GLL polynomial through `in` at the points of order
// (n-1) (project_points_to_target_polynomial.hpp).
inline std::vector<std::array<double, 3>> ProjectPoints(size_t m, size_t n,
                                                        const std::vector<std::array<double, 3>>& in) {
    const auto from = GenerateGLLPoints(m - 1), to = GenerateGLLPoints(n - 1);
    std::vector<std::array<double, 3>> out(n, {0., 0., 0.});
    for (size_t o = 0; o < n; ++o) {
        const auto w = LagrangeWeights(to[o], from);
        for (size_t i = 0; i < m; ++i)
            for (int d = 0; d < 3; ++d) out[o][d] += w[i] * in[i][d];
    }
    return out;
}

}  // namespace math

namespace components {

enum class ReferenceAxisOrientation { X, Z };

// src/interfaces/components/beam_input.hpp
struct ReferenceAxis {
    std::vector<double> coordinate_grid;
    std::vector<std::array<double, 3>> coordinates;
    std::vector<double> twist_grid;
    std::vector<double> twist;   // degrees
};

struct Section {
    double location;
    math::M6 mass_matrix, stiffness_matrix;
    Section(double loc, const math::M6& m, const math::M6& k) : location(loc), mass_matrix(m), stiffness_matrix(k) {
        if (loc < 0. || loc > 1.) throw std::invalid_argument("section location must be in [0, 1]");
    }
};

struct Root {
    bool prescribe_root_motion = false;
    std::array<double, 7> position{0., 0., 0., 1., 0., 0., 0.};
    std::array<double, 6> velocity{};
    std::array<double, 6> acceleration{};
};

struct BeamInput {
    size_t element_order = 10;
    size_t section_refinement = 0;
    ReferenceAxis ref_axis;
    Root root;
    std::vector<Section> sections;
};

// src/interfaces/node_data.hpp: one node's motion out and loads in
struct NodeData {
    size_t id;
    std::array<double, 7> position{0., 0., 0., 1., 0., 0., 0.};
    std::array<double, 7> displacement{0., 0., 0., 1., 0., 0., 0.};
    std::array<double, 6> velocity{};
    std::array<double, 6> acceleration{};
    std::array<double, 6> loads{};
    explicit NodeData(size_t i) : id(i) {}
    void ClearLoads() { loads = {0., 0., 0., 0., 0., 0.}; }
};

// The rotation taking a Z-up (WindIO) reference axis to the X axis.
inline std::array<double, 4> ZToX() { return RotationVectorToQuaternion({0., std::numbers::pi / 2., 0.}); }

// src/interfaces/components/beam_builder.cpp
class BeamBuilder {
public:
    BeamBuilder& SetElementOrder(size_t order) { input_.element_order = order; return *this; }
    BeamBuilder& SetSectionRefinement(size_t r) { input_.section_refinement = r; return *this; }
    BeamBuilder& AddRefAxisPoint(double s, const std::array<double, 3>& c,
                                 ReferenceAxisOrientation o = ReferenceAxisOrientation::X) {
        input_.ref_axis.coordinate_grid.push_back(s);
        input_.ref_axis.coordinates.push_back(o == ReferenceAxisOrientation::X
                                                  ? c : RotateVectorByQuaternion(ZToX(), c));
        return *this;
    }
    BeamBuilder& AddRefAxisTwist(double s, double twist) {
        input_.ref_axis.twist_grid.push_back(s);
        input_.ref_axis.twist.push_back(twist);
        return *this;
    }
    BeamBuilder& PrescribedRootMotion(bool on) { input_.root.prescribe_root_motion = on; return *this; }
    BeamBuilder& SetRootPosition(const std::array<double, 7>& p) { input_.root.position = p; return *this; }
    BeamBuilder& SetRootVelocity(const std::array<double, 6>& v) { input_.root.velocity = v; return *this; }
    BeamBuilder& SetRootAcceleration(const std::array<double, 6>& a) { input_.root.acceleration = a; return *this; }
    BeamBuilder& AddSection(double s, const math::M6& mass, const math::M6& stiffness,
                            ReferenceAxisOrientation o = ReferenceAxisOrientation::X) {
        if (o == ReferenceAxisOrientation::X)
            input_.sections.emplace_back(s, mass, stiffness);
        else
            input_.sections.emplace_back(s, math::RotateMatrix6(mass, ZToX()), math::RotateMatrix6(stiffness, ZToX()));
        return *this;
    }
    const BeamInput& Input() const { return input_; }

private:
    BeamInput input_;
};

// src/interfaces/components/beam.cpp: the blade as one beam element of the
// requested order on GLL nodes fitted to the reference axis, trapezoidal
// quadrature at the section stations, placed at the root.
class Beam {
public:
    static constexpr size_t kMaxGeometryPoints = 10;
    static constexpr size_t invalid_id = static_cast<size_t>(-1);
    std::vector<NodeData> nodes;
    size_t beam_element_id = 0;
    size_t prescribed_root_constraint_id = invalid_id;

    Beam(const BeamInput& in, Model& model) {
        if (in.ref_axis.coordinate_grid.size() < 2 || in.ref_axis.coordinates.size() < 2)
            throw std::invalid_argument("at least two reference axis points are required");
        if (in.ref_axis.coordinate_grid.size() != in.ref_axis.coordinates.size())
            throw std::invalid_argument("reference axis grid and coordinates differ in size");
        if (in.sections.empty()) throw std::invalid_argument("at least one section is required");
        if (in.element_order < 1) throw std::invalid_argument("element order must be at least 1");
        node_xi_ = math::GenerateGLLPoints(in.element_order);
        const size_t n_nodes = in.element_order + 1;
        const size_t n_geo = std::min({in.ref_axis.coordinate_grid.size(), n_nodes, kMaxGeometryPoints});
        std::vector<std::array<double, 3>> coords;
        if (n_geo < n_nodes) {
            const auto geo = math::FitNodes(math::GenerateGLLPoints(n_geo - 1), in.ref_axis.coordinate_grid,
                                            in.ref_axis.coordinates);
            coords = math::ProjectPoints(n_geo, n_nodes, geo);
        } else {
            coords = math::FitNodes(node_xi_, in.ref_axis.coordinate_grid, in.ref_axis.coordinates);
        }
        // tangents: derivative of the node polynomial at the nodes, normalised
        std::vector<std::array<double, 3>> tangents(n_nodes, {0., 0., 0.});
        for (size_t a = 0; a < n_nodes; ++a) {
            const auto dw = math::LagrangeDerivWeights(node_xi_[a], node_xi_);
            for (size_t b = 0; b < n_nodes; ++b)
                for (int d = 0; d < 3; ++d) tangents[a][d] += dw[b] * coords[b][d];
            tangents[a] = math::Unit(tangents[a]);
        }
        std::vector<size_t> ids;
        for (size_t k = 0; k < n_nodes; ++k) {
            const auto q = math::TangentTwistToQuaternion(tangents[k], 0.);
            ids.push_back(model.AddNode()
                              .SetElemLocation((node_xi_[k] + 1.) / 2.)
                              .SetPosition(coords[k][0], coords[k][1], coords[k][2], q[0], q[1], q[2], q[3])
                              .Build());
            nodes.emplace_back(ids.back());
        }
        const auto sections = BuildSections(in);
        std::vector<double> grid;
        for (const auto& s : sections) grid.push_back(s.position);
        const auto quad = math::CreateTrapezoidalQuadrature(grid);
        beam_element_id = model.AddBeamElement(ids, sections, quad);
        // place at the root
        const std::array<double, 3> p{in.root.position[0], in.root.position[1], in.root.position[2]};
        model.TranslateBeam(beam_element_id, p);
        model.RotateBeamAboutPoint(beam_element_id, {in.root.position[3], in.root.position[4],
                                                     in.root.position[5], in.root.position[6]}, p);
        model.SetBeamVelocityAboutPoint(beam_element_id, in.root.velocity, p);
        model.SetBeamAccelerationAboutPoint(beam_element_id, in.root.acceleration,
                                            {in.root.velocity[3], in.root.velocity[4], in.root.velocity[5]}, p);
        if (in.root.prescribe_root_motion) prescribed_root_constraint_id = model.AddPrescribedBC(ids.front());
    }

    // Distributes a point load at s in [0, 1] over the nodes with the weights
    // the reference's Beam::AddPointLoad uses (its GetNodeWeights returns the
    // Lagrange derivative weights at s, beam.cpp:24-41); kept as it is so that
    // callers see the same nodal loads.
    void AddPointLoad(double s, const std::array<double, 6>& loads) {
        if (s < 0. || s > 1.) throw std::invalid_argument("invalid load position");
        const auto w = math::LagrangeDerivWeights(2. * s - 1., node_xi_);
        for (size_t k = 0; k < nodes.size(); ++k)
            for (int c = 0; c < 6; ++c) nodes[k].loads[c] += w[k] * loads[c];
    }
    void ClearLoads() {
        for (auto& n : nodes) n.ClearLoads();
    }

private:
    std::vector<double> node_xi_;

    // Sections rotated by the interpolated twist about x, with optional linear
    // refinement between stations (Beam::BuildBeamSections).
    static std::vector<BeamSection> BuildSections(const BeamInput& in) {
        auto twist_q = [&](double s) {
            const double tw = math::LinearInterp(s, in.ref_axis.twist_grid, in.ref_axis.twist);
            return RotationVectorToQuaternion({tw * std::numbers::pi / 180., 0., 0.});
        };
        std::vector<BeamSection> out;
        const auto& s0 = in.sections.front();
        out.emplace_back(s0.location, math::RotateMatrix6(s0.mass_matrix, twist_q(s0.location)),
                         math::RotateMatrix6(s0.stiffness_matrix, twist_q(s0.location)));
        for (size_t i = 1; i < in.sections.size(); ++i) {
            const auto& L = in.sections[i - 1];
            const auto& R = in.sections[i];
            for (size_t r = 0; r < in.section_refinement; ++r) {
                const double al = static_cast<double>(r + 1) / static_cast<double>(in.section_refinement + 1);
                math::M6 m{}, k{};
                for (int a = 0; a < 6; ++a)
                    for (int b = 0; b < 6; ++b) {
                        m[a][b] = (1. - al) * L.mass_matrix[a][b] + al * R.mass_matrix[a][b];
                        k[a][b] = (1. - al) * L.stiffness_matrix[a][b] + al * R.stiffness_matrix[a][b];
                    }
                // the reference takes the twist of the right station here
                const auto q = twist_q(R.location);
                out.emplace_back((1. - al) * L.location + al * R.location, math::RotateMatrix6(m, q),
                                 math::RotateMatrix6(k, q));
            }
            const auto q = twist_q(R.location);
            out.emplace_back(R.location, math::RotateMatrix6(R.mass_matrix, q),
                             math::RotateMatrix6(R.stiffness_matrix, q));
        }
        return out;
    }
};

// src/interfaces/components/solution_input.hpp
struct SolutionInput {
    std::array<double, 3> gravity{0., 0., 0.};
    bool dynamic_solve = true;
    double time_step = 0.01;
    double rho_inf = 0.;
    size_t max_iter = 5;
    double absolute_error_tolerance = 1e-5;
    double relative_error_tolerance = 1e-3;
    std::string output_file_path;
    StepParameters Parameters() const {
        return StepParameters(dynamic_solve, max_iter, time_step, rho_inf, absolute_error_tolerance,
                              relative_error_tolerance);
    }
};

// src/interfaces/components/solution_builder.hpp
class SolutionBuilder {
public:
    SolutionBuilder& EnableDynamicSolve() { in_.dynamic_solve = true; return *this; }
    SolutionBuilder& EnableStaticSolve() { in_.dynamic_solve = false; return *this; }
    SolutionBuilder& SetTimeStep(double h) { in_.time_step = h; return *this; }
    SolutionBuilder& SetDampingFactor(double rho) { in_.rho_inf = rho; return *this; }
    SolutionBuilder& SetGravity(const std::array<double, 3>& g) { in_.gravity = g; return *this; }
    SolutionBuilder& SetMaximumNonlinearIterations(size_t n) { in_.max_iter = n; return *this; }
    SolutionBuilder& SetAbsoluteErrorTolerance(double t) { in_.absolute_error_tolerance = t; return *this; }
    SolutionBuilder& SetRelativeErrorTolerance(double t) { in_.relative_error_tolerance = t; return *this; }
    SolutionBuilder& SetOutputFile(const std::string& p) { in_.output_file_path = p; return *this; }
    const SolutionInput& Input() const { return in_; }

private:
    SolutionInput in_;
};

}  // namespace components

// src/interfaces/blade/blade_interface.hpp: a blade with loads in and motion
// out per step, a saved state for predictor-corrector coupling, and the root
// motion when it is prescribed.
class BladeInterface {
public:
    BladeInterface(const Context& ctx, const components::SolutionInput& sol, const components::BeamInput& blade)
        : ctx_(ctx), model_(sol.gravity), blade_(blade, model_), parameters_(sol.Parameters()) {
        auto [state, elements, constraints, solver] = model_.CreateSystemWithSolver(ctx_);
        state_ = std::make_unique<State>(state);
        elements_ = std::make_unique<Elements>(elements);
        constraints_ = std::make_unique<Constraints>(constraints);
        solver_ = std::make_unique<Solver>(solver);
        const int id = solver_->model()->id;
        saved_ = kyn_model_clone(ctx_.get(), id);   // state_save (CloneState)
        check(ctx_.get(), saved_);
        loads_.assign(solver_->model()->info.num_nodes * 6, 0.);
        GetMotion();
    }
    BladeInterface(const BladeInterface&) = delete;
    BladeInterface& operator=(const BladeInterface&) = delete;
    BladeInterface(BladeInterface&& o) noexcept
        : ctx_(o.ctx_), model_(std::move(o.model_)), blade_(std::move(o.blade_)),
          parameters_(o.parameters_), state_(std::move(o.state_)), elements_(std::move(o.elements_)),
          constraints_(std::move(o.constraints_)), solver_(std::move(o.solver_)), saved_(o.saved_),
          loads_(std::move(o.loads_)) {
        o.saved_ = -1;
    }
    ~BladeInterface() {
        if (saved_ >= 0) kyn_model_destroy(ctx_.get(), saved_);
    }

    components::Beam& Blade() { return blade_; }

    // Node loads -> state.f, one step, motion of the nodes back (false: the
    // Newton loop reached max_iter, as the reference's Step()).
    bool Step() {
        for (const auto& n : blade_.nodes)
            for (int c = 0; c < 6; ++c) loads_[n.id * 6 + c] = n.loads[c];
        state_->SetExternalForces(loads_);
        if (!kynema_b200::Step(parameters_, *solver_, *elements_, *state_, *constraints_)) return false;
        GetMotion();
        return true;
    }
    void SaveState() { check(ctx_.get(), kyn_state_copy(ctx_.get(), saved_, solver_->model()->id)); }
    void RestoreState() {
        check(ctx_.get(), kyn_state_copy(ctx_.get(), solver_->model()->id, saved_));
        GetMotion();
    }
    void SetRootDisplacement(const std::array<double, 7>& u) const {
        if (blade_.prescribed_root_constraint_id == components::Beam::invalid_id)
            throw std::runtime_error("prescribed root motion was not enabled");
        constraints_->UpdateDisplacement(blade_.prescribed_root_constraint_id, u);
    }

private:
    void GetMotion() {
        const auto x = state_->Get(KYN_FIELD_X), q = state_->q(), v = state_->v(), vd = state_->vd();
        for (auto& n : blade_.nodes) {
            for (int c = 0; c < 7; ++c) {
                n.position[c] = x[n.id * 7 + c];
                n.displacement[c] = q[n.id * 7 + c];
            }
            for (int c = 0; c < 6; ++c) {
                n.velocity[c] = v[n.id * 6 + c];
                n.acceleration[c] = vd[n.id * 6 + c];
            }
        }
    }

    Context ctx_;
    Model model_;
    components::Beam blade_;
    StepParameters parameters_;
    std::unique_ptr<State> state_;
    std::unique_ptr<Elements> elements_;
    std::unique_ptr<Constraints> constraints_;
    std::unique_ptr<Solver> solver_;
    int saved_ = -1;
    std::vector<double> loads_;
};

// src/interfaces/blade/blade_interface_builder.hpp
class BladeInterfaceBuilder {
public:
    components::SolutionBuilder& Solution() { return solution_; }
    components::BeamBuilder& Blade() { return blade_; }
    BladeInterface Build(const Context& ctx = Context(0)) const {
        return BladeInterface(ctx, solution_.Input(), blade_.Input());
    }

private:
    components::SolutionBuilder solution_;
    components::BeamBuilder blade_;
};

// ---- sectional properties of a hollow circular tube ---------------------------------
// src/elements/beams/generate_sectional_properties.hpp and
// hollow_circle_properties.hpp: the 6x6 stiffness and mass matrices of a
// section about its reference point (the beam axis along z of the section
// frame, WindIO convention), from its stiffnesses, inertias, offsets of the
// elastic centre, shear centre and centre of gravity, and principal-axis angles.
namespace beams {

inline math::M6 GenerateStiffnessMatrix(double EA, double EI_x, double EI_y, double GKt, double GA, double kxs,
                                        double kys, double x_C, double y_C, double theta_p, double x_S,
                                        double y_S, double theta_s) {
    const double cp = std::cos(theta_p), sp = std::sin(theta_p);
    const double cs = std::cos(theta_s), ss = std::sin(theta_s);
    const double bxx = EI_x * cp * cp + EI_y * sp * sp;
    const double byy = EI_x * sp * sp + EI_y * cp * cp;
    const double bxy = (EI_y - EI_x) * sp * cp;
    const double sxx = GA * (kxs * cs * cs + kys * ss * ss);
    const double syy = GA * (kxs * ss * ss + kys * cs * cs);
    const double sxy = GA * (kys - kxs) * ss * cs;
    math::M6 k{};
    k[0][0] = sxx;
    k[0][1] = k[1][0] = -sxy;
    k[1][1] = syy;
    k[2][2] = EA;
    k[2][3] = k[3][2] = EA * y_C;
    k[2][4] = k[4][2] = -EA * x_C;
    k[3][3] = bxx + EA * y_C * y_C;
    k[3][4] = k[4][3] = -bxy - EA * x_C * y_C;
    k[4][4] = byy + EA * x_C * x_C;
    k[0][5] = k[5][0] = -sxx * y_S - sxy * x_S;
    k[1][5] = k[5][1] = sxy * y_S + syy * x_S;
    k[5][5] = GKt + sxx * y_S * y_S + 2. * sxy * x_S * y_S + syy * x_S * x_S;
    return k;
}

inline math::M6 GenerateMassMatrix(double m, double I_x, double I_y, double I_p, double x_G = 0., double y_G = 0.,
                                   double theta_i = 0.) {
    const double ci = std::cos(theta_i), si = std::sin(theta_i);
    const double ixx = I_x * ci * ci + I_y * si * si;
    const double iyy = I_x * si * si + I_y * ci * ci;
    const double ixy = (I_y - I_x) * si * ci;
    math::M6 M{};
    M[0][0] = M[1][1] = M[2][2] = m;
    M[0][5] = M[5][0] = -m * y_G;
    M[1][5] = M[5][1] = m * x_G;
    M[2][3] = M[3][2] = m * y_G;
    M[2][4] = M[4][2] = -m * x_G;
    M[3][3] = ixx + m * y_G * y_G;
    M[3][4] = M[4][3] = -ixy - m * x_G * y_G;
    M[4][4] = iyy + m * x_G * x_G;
    M[5][5] = I_p + m * (x_G * x_G + y_G * y_G);
    return M;
}

struct HollowCircleProperties {
    double area, Ixx, Iyy, J, kx, ky;
};

// Area, second moments and polar moment of a tube of outer diameter D and
// wall t, Timoshenko shear factor 6 (1 + nu) / (7 + 6 nu).
inline HollowCircleProperties CalculateHollowCircleProperties(double D, double t, double nu = 0.33) {
    if (t >= D / 2.) throw std::invalid_argument("wall thickness must be less than the outer radius");
    const double ro = D / 2., ri = ro - t;
    const double area = std::numbers::pi * (ro * ro - ri * ri);
    const double I = std::numbers::pi * (std::pow(ro, 4) - std::pow(ri, 4)) / 4.;
    const double k = 6. * (1. + nu) / (7. + 6. * nu);
    return {area, I, I, 2. * I, k, k};
}

inline BeamSection GenerateHollowCircleSection(double s, double E, double G, double rho, double D, double t,
                                               double nu, double x_C = 0., double y_C = 0., double theta_p = 0.,
                                               double x_S = 0., double y_S = 0., double theta_s = 0.,
                                               double x_G = 0., double y_G = 0., double theta_i = 0.) {
    const auto p = CalculateHollowCircleProperties(D, t, nu);
    const double Ix = rho * p.Ixx, Iy = rho * p.Iyy;
    return {s, GenerateMassMatrix(rho * p.area, Ix, Iy, Ix + Iy, x_G, y_G, theta_i),
            GenerateStiffnessMatrix(E * p.area, E * p.Ixx, E * p.Iyy, G * p.J, G * p.area, p.kx, p.ky, x_C, y_C,
                                    theta_p, x_S, y_S, theta_s)};
}

}  // namespace beams

// ---- turbine: tower, drive train, hub, blades -----------------------------------------
namespace components {

// src/interfaces/components/turbine_input.hpp
struct TurbineInput {
    std::vector<BeamInput> blades;
    BeamInput tower;
    math::M6 yaw_bearing_inertia_matrix{};
    math::M6 hub_inertia_matrix{};
    std::array<double, 7> tower_base_position{0., 0., 0., 1., 0., 0., 0.};
    double tower_axis_to_rotor_apex = 0.;
    double tower_top_to_rotor_apex = 0.;
    double rotor_apex_to_hub = 0.;
    double hub_diameter = 1e-7;
    double nacelle_yaw_angle = 0.;
    double shaft_tilt_angle = 0.;
    double cone_angle = 0.;
    double blade_pitch_angle = 0.;
    double azimuth_angle = 0.;
    double rotor_speed = 0.;
};

struct ConstraintData {
    size_t id;
};

// src/interfaces/components/turbine.cpp: the blades and the tower as beam
// components; a yaw bearing at the tower top (nacelle mass), a shaft base, an
// azimuth node, a hub (hub mass) and one apex node per blade, placed by the
// turbine's geometry (tower axis to z, blades to z at the hub radius, cone,
// azimuth spacing, shaft tilt, rotor apex); the joints tower top -> yaw
// bearing (RotationControl about z, yaw), yaw bearing -> shaft base (rigid),
// shaft base -> azimuth (revolute about the shaft axis, generator torque),
// azimuth -> hub (rigid), hub -> apex (rigid) and blade root -> apex
// (RotationControl about the pitch axis); initial pitch, yaw and tower-base
// displacements, a PrescribedBC at the tower base and the rotor's initial
// speed about the shaft.  The constraints read blade_pitch_control,
// yaw_control and torque_control before every step, so a Turbine stays where
// it was built.
class Turbine {
public:
    static constexpr size_t invalid_id = static_cast<size_t>(-1);
    static constexpr double kMinHubDiameter = 1e-8;
    static constexpr double kZeroTolerance = 1e-12;

    std::vector<Beam> blades;
    Beam tower;
    size_t hub_mass_element_id = invalid_id;
    size_t yaw_bearing_mass_element_id = invalid_id;
    std::vector<NodeData> apex_nodes;
    NodeData hub_node{invalid_id};
    NodeData azimuth_node{invalid_id};
    NodeData shaft_base_node{invalid_id};
    NodeData yaw_bearing_node{invalid_id};
    ConstraintData tower_base{invalid_id};
    ConstraintData tower_top_to_yaw_bearing{invalid_id};
    ConstraintData yaw_bearing_to_shaft_base{invalid_id};
    ConstraintData shaft_base_to_azimuth{invalid_id};
    ConstraintData azimuth_to_hub{invalid_id};
    std::vector<ConstraintData> blade_pitch;
    std::vector<ConstraintData> apex_to_hub;
    std::vector<double> blade_pitch_control;
    double torque_control = 0.;
    double yaw_control = 0.;

    Turbine(const TurbineInput& in, Model& model)
        : blades(CreateBlades(in.blades, model)), tower(in.tower, model),
          blade_pitch_control(in.blades.size(), in.blade_pitch_angle) {
        if (in.hub_diameter <= kMinHubDiameter) throw std::invalid_argument("hub diameter must be > 1e-8");
        if (in.rotor_speed < 0.) throw std::invalid_argument("rotor speed must be >= 0");
        if (blades.empty()) throw std::invalid_argument("a turbine needs at least one blade");
        PositionNodes(in, model);
        yaw_bearing_mass_element_id = model.AddMassElement(yaw_bearing_node.id, in.yaw_bearing_inertia_matrix);
        hub_mass_element_id = model.AddMassElement(hub_node.id, in.hub_inertia_matrix);
        AddConstraints(in, model);
        SetInitialDisplacements(in, model);
        SetInitialRotorVelocity(in, model);
    }
    Turbine(const Turbine&) = delete;
    Turbine& operator=(const Turbine&) = delete;

private:
    std::vector<size_t> tower_node_ids_, nacelle_node_ids_, rotor_node_ids_, blade_node_ids_;

    static std::vector<Beam> CreateBlades(const std::vector<BeamInput>& inputs, Model& model) {
        std::vector<Beam> out;
        for (const auto& b : inputs) out.emplace_back(b, model);
        return out;
    }

    void PositionNodes(const TurbineInput& in, Model& model) {
        const std::array<double, 3> origin{0., 0., 0.};
        const double blade_angle = 2. * std::numbers::pi / static_cast<double>(blades.size());
        const auto q_x_to_z = RotationVectorToQuaternion({0., -std::numbers::pi / 2., 0.});
        const auto q_cone = RotationVectorToQuaternion({0., -in.cone_angle, 0.});
        model.RotateBeamAboutPoint(tower.beam_element_id, q_x_to_z, origin);
        const auto& top = model.GetNode(tower.nodes.back().id);
        const std::array<double, 3> apex{top.x0[0] - in.tower_axis_to_rotor_apex, top.x0[1],
                                         top.x0[2] + in.tower_top_to_rotor_apex};
        CreateIntermediateNodes(in, model);
        for (size_t b = 0; b < blades.size(); ++b) {
            std::vector<size_t> ids;
            for (const auto& n : blades[b].nodes) ids.push_back(n.id);
            for (size_t id : ids) {
                model.GetNode(id).RotateAboutPoint(q_x_to_z, origin);
                model.GetNode(id).Translate({0., 0., in.hub_diameter / 2.});
            }
            ids.push_back(apex_nodes[b].id);
            const auto q_az = RotationVectorToQuaternion({static_cast<double>(b) * blade_angle, 0., 0.});
            for (size_t id : ids) {
                model.GetNode(id).RotateAboutPoint(q_cone, origin);
                model.GetNode(id).RotateAboutPoint(q_az, origin);
            }
        }
        const auto q_tilt = RotationVectorToQuaternion({0., in.shaft_tilt_angle, 0.});
        for (size_t id : rotor_node_ids_) {
            model.GetNode(id).RotateAboutPoint(q_tilt, origin);
            model.GetNode(id).Translate(apex);
        }
    }

    void CreateIntermediateNodes(const TurbineInput& in, Model& model) {
        const double shaft_length = in.tower_axis_to_rotor_apex / std::cos(in.shaft_tilt_angle);
        const auto top = model.GetNode(tower.nodes.back().id).x0;
        hub_node = NodeData(model.AddNode().SetPosition(-in.rotor_apex_to_hub, 0., 0., 1., 0., 0., 0.).Build());
        azimuth_node = NodeData(model.AddNode().SetPosition(shaft_length, 0., 0., 1., 0., 0., 0.).Build());
        shaft_base_node = NodeData(model.AddNode().SetPosition(shaft_length, 0., 0., 1., 0., 0., 0.).Build());
        yaw_bearing_node = NodeData(model.AddNode().SetPosition(top[0], top[1], top[2], 1., 0., 0., 0.).Build());
        for (size_t b = 0; b < blades.size(); ++b)
            apex_nodes.emplace_back(model.AddNode().SetPosition(0., 0., 0., 1., 0., 0., 0.).Build());
        for (const auto& n : tower.nodes) tower_node_ids_.push_back(n.id);
        for (size_t b = 0; b < blades.size(); ++b) {
            for (const auto& n : blades[b].nodes) blade_node_ids_.push_back(n.id);
            blade_node_ids_.push_back(apex_nodes[b].id);
        }
        rotor_node_ids_ = {hub_node.id, azimuth_node.id, shaft_base_node.id};
        rotor_node_ids_.insert(rotor_node_ids_.end(), blade_node_ids_.begin(), blade_node_ids_.end());
        nacelle_node_ids_ = {yaw_bearing_node.id, shaft_base_node.id, azimuth_node.id, hub_node.id};
        nacelle_node_ids_.insert(nacelle_node_ids_.end(), blade_node_ids_.begin(), blade_node_ids_.end());
    }

    void AddConstraints(const TurbineInput& in, Model& model) {
        for (size_t b = 0; b < blades.size(); ++b) {
            const auto& apex = model.GetNode(apex_nodes[b].id);
            const auto& root = model.GetNode(blades[b].nodes[0].id);
            const std::array<double, 3> pitch_axis{root.x0[0] - apex.x0[0], root.x0[1] - apex.x0[1],
                                                   root.x0[2] - apex.x0[2]};
            blade_pitch.push_back({model.AddRotationControl({root.id, apex.id}, pitch_axis, &blade_pitch_control[b])});
            apex_to_hub.push_back({model.AddRigidJointConstraint({hub_node.id, apex_nodes[b].id})});
        }
        azimuth_to_hub = {model.AddRigidJointConstraint({azimuth_node.id, hub_node.id})};
        const std::array<double, 3> shaft_axis{-std::cos(in.shaft_tilt_angle), 0., std::sin(in.shaft_tilt_angle)};
        shaft_base_to_azimuth = {
            model.AddRevoluteJointConstraint({shaft_base_node.id, azimuth_node.id}, shaft_axis, &torque_control)};
        yaw_bearing_to_shaft_base = {model.AddRigidJointConstraint({yaw_bearing_node.id, shaft_base_node.id})};
        yaw_control = in.nacelle_yaw_angle;
        tower_top_to_yaw_bearing = {
            model.AddRotationControl({tower.nodes.back().id, yaw_bearing_node.id}, {0., 0., 1.}, &yaw_control)};
    }

    // Node::RotateDisplacementAboutPoint (src/model/node.hpp:152-187)
    static void RotateDisplacement(Node& n, const std::array<double, 4>& q, const std::array<double, 3>& p) {
        const auto d = n.DisplacedPosition();
        const auto r = RotateVectorByQuaternion(q, {d[0] - p[0], d[1] - p[1], d[2] - p[2]});
        for (int k = 0; k < 3; ++k) n.u[k] = r[k] + p[k] - n.x0[k];
        const auto qn = QuaternionCompose(q, {n.u[3], n.u[4], n.u[5], n.u[6]});
        for (int k = 0; k < 4; ++k) n.u[3 + k] = qn[k];
    }

    void SetInitialDisplacements(const TurbineInput& in, Model& model) {
        for (size_t b = 0; b < blades.size(); ++b) {
            const auto& root = model.GetNode(blades[b].nodes.front().id);
            const auto& apex = model.GetNode(apex_nodes[b].id);
            const auto axis = math::Unit({root.x0[0] - apex.x0[0], root.x0[1] - apex.x0[1], root.x0[2] - apex.x0[2]});
            const auto q_pitch = RotationVectorToQuaternion(
                {in.blade_pitch_angle * axis[0], in.blade_pitch_angle * axis[1], in.blade_pitch_angle * axis[2]});
            const std::array<double, 3> center{apex.x0[0], apex.x0[1], apex.x0[2]};
            for (const auto& n : blades[b].nodes) RotateDisplacement(model.GetNode(n.id), q_pitch, center);
        }
        if (std::abs(in.nacelle_yaw_angle) > kZeroTolerance) {
            const auto& top = model.GetNode(tower.nodes.back().id);
            const std::array<double, 3> center{top.x0[0], top.x0[1], top.x0[2]};
            const auto q_yaw = RotationVectorToQuaternion({0., 0., in.nacelle_yaw_angle});
            for (size_t id : nacelle_node_ids_) RotateDisplacement(model.GetNode(id), q_yaw, center);
        }
        auto& base = model.GetNode(tower.nodes.front().id);
        const std::array<double, 3> ref{base.x0[0], base.x0[1], base.x0[2]};
        const std::array<double, 3> d{in.tower_base_position[0] - ref[0], in.tower_base_position[1] - ref[1],
                                      in.tower_base_position[2] - ref[2]};
        const std::array<double, 4> qb{in.tower_base_position[3], in.tower_base_position[4],
                                       in.tower_base_position[5], in.tower_base_position[6]};
        const bool identity = std::abs(qb[0] - 1.) <= kZeroTolerance && std::abs(qb[1]) <= kZeroTolerance &&
                              std::abs(qb[2]) <= kZeroTolerance && std::abs(qb[3]) <= kZeroTolerance;
        if (std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]) > kZeroTolerance || !identity) {
            std::vector<size_t> all = tower_node_ids_;
            all.insert(all.end(), nacelle_node_ids_.begin(), nacelle_node_ids_.end());
            for (size_t id : all) {
                auto& n = model.GetNode(id);
                RotateDisplacement(n, qb, ref);
                for (int k = 0; k < 3; ++k) n.u[k] += d[k];
            }
        }
        tower_base = {model.AddPrescribedBC(base.id, base.u)};
    }

    void SetInitialRotorVelocity(const TurbineInput& in, Model& model) {
        const auto hp = model.GetNode(hub_node.id).DisplacedPosition();
        const auto sp = model.GetNode(shaft_base_node.id).DisplacedPosition();
        const auto axis = math::Unit({hp[0] - sp[0], hp[1] - sp[1], hp[2] - sp[2]});
        std::vector<size_t> ids{hub_node.id, azimuth_node.id};
        for (size_t b = 0; b < blades.size(); ++b) {
            for (const auto& n : blades[b].nodes) ids.push_back(n.id);
            ids.push_back(apex_nodes[b].id);
        }
        const std::array<double, 6> vel{0., 0., 0., in.rotor_speed * axis[0], in.rotor_speed * axis[1],
                                        in.rotor_speed * axis[2]};
        for (size_t id : ids) model.GetNode(id).SetVelocityAboutPoint(vel, {hp[0], hp[1], hp[2]});
    }
};

// src/interfaces/components/turbine_builder.hpp
class TurbineBuilder {
public:
    BeamBuilder& Blade(size_t i) {
        if (i >= blades_.size()) blades_.resize(i + 1);
        return blades_[i];
    }
    BeamBuilder& Tower() { return tower_; }
    TurbineBuilder& SetYawBearingInertiaMatrix(const math::M6& m) { in_.yaw_bearing_inertia_matrix = m; return *this; }
    TurbineBuilder& SetHubInertiaMatrix(const math::M6& m) { in_.hub_inertia_matrix = m; return *this; }
    TurbineBuilder& SetTowerBasePosition(const std::array<double, 7>& p) { in_.tower_base_position = p; return *this; }
    TurbineBuilder& SetTowerAxisToRotorApex(double d) { in_.tower_axis_to_rotor_apex = d; return *this; }
    TurbineBuilder& SetTowerTopToRotorApex(double h) { in_.tower_top_to_rotor_apex = h; return *this; }
    TurbineBuilder& SetRotorApexToHub(double d) { in_.rotor_apex_to_hub = d; return *this; }
    TurbineBuilder& SetHubDiameter(double d) { in_.hub_diameter = d; return *this; }
    TurbineBuilder& SetShaftTiltAngle(double a) { in_.shaft_tilt_angle = a; return *this; }
    TurbineBuilder& SetNacelleYawAngle(double a) { in_.nacelle_yaw_angle = a; return *this; }
    TurbineBuilder& SetConeAngle(double a) { in_.cone_angle = a; return *this; }
    TurbineBuilder& SetBladePitchAngle(double a) { in_.blade_pitch_angle = a; return *this; }
    TurbineBuilder& SetAzimuthAngle(double a) { in_.azimuth_angle = a; return *this; }
    TurbineBuilder& SetRotorSpeed(double w) { in_.rotor_speed = w; return *this; }
    TurbineInput Input() const {
        TurbineInput in = in_;
        in.blades.clear();
        for (const auto& b : blades_) in.blades.push_back(b.Input());
        in.tower = tower_.Input();
        return in;
    }

private:
    TurbineInput in_;
    std::vector<BeamBuilder> blades_;
    BeamBuilder tower_;
};

}  // namespace components

// src/interfaces/turbine/turbine_interface.hpp: the turbine with node loads in
// (state.f) and the motion of the blade and tower nodes out after each step,
// a saved state for predictor-corrector coupling.  The aerodynamics, the
// controller library and the NetCDF outputs of the reference's interface are
// outside this path.
class TurbineInterface {
public:
    TurbineInterface(const Context& ctx, const components::SolutionInput& sol, const components::TurbineInput& in)
        : ctx_(ctx), model_(sol.gravity), turbine_(in, model_), parameters_(sol.Parameters()) {
        auto [state, elements, constraints, solver] = model_.CreateSystemWithSolver(ctx_);
        state_ = std::make_unique<State>(state);
        elements_ = std::make_unique<Elements>(elements);
        constraints_ = std::make_unique<Constraints>(constraints);
        solver_ = std::make_unique<Solver>(solver);
        saved_ = kyn_model_clone(ctx_.get(), solver_->model()->id);
        check(ctx_.get(), saved_);
        loads_.assign(solver_->model()->info.num_nodes * 6, 0.);
        GetMotion();
    }
    TurbineInterface(const TurbineInterface&) = delete;
    TurbineInterface& operator=(const TurbineInterface&) = delete;
    ~TurbineInterface() {
        if (saved_ >= 0) kyn_model_destroy(ctx_.get(), saved_);
    }

    components::Turbine& Turbine() { return turbine_; }
    const Model& GetModel() const { return model_; }
    const Solver& GetSolver() const { return *solver_; }

    // Node loads of the blades and the tower -> state.f, the controls into
    // their constraints, one step, motion back (false: max_iter reached).
    bool Step() {
        std::fill(loads_.begin(), loads_.end(), 0.);
        auto put = [&](const components::Beam& b) {
            for (const auto& n : b.nodes)
                for (int c = 0; c < 6; ++c) loads_[n.id * 6 + c] = n.loads[c];
        };
        for (const auto& b : turbine_.blades) put(b);
        put(turbine_.tower);
        state_->SetExternalForces(loads_);
        if (!kynema_b200::Step(parameters_, *solver_, *elements_, *state_, *constraints_)) return false;
        GetMotion();
        return true;
    }
    void SaveState() { check(ctx_.get(), kyn_state_copy(ctx_.get(), saved_, solver_->model()->id)); }
    void RestoreState() {
        check(ctx_.get(), kyn_state_copy(ctx_.get(), solver_->model()->id, saved_));
        GetMotion();
    }
    // Rotation of the shaft joint about its axis, wrapped to [0, 2 pi), and the
    // rotor speed about it (TurbineInterface::CalculateAzimuthAngle /
    // CalculateRotorSpeed, src/interfaces/turbine/turbine_interface.cpp:206-222)
    double CalculateAzimuthAngle() const {
        double azimuth = constraints_->output()[turbine_.shaft_base_to_azimuth.id * 3];
        azimuth = std::fmod(azimuth, 2. * std::numbers::pi);
        return azimuth < 0. ? azimuth + 2. * std::numbers::pi : azimuth;
    }
    double CalculateRotorSpeed() const { return constraints_->output()[turbine_.shaft_base_to_azimuth.id * 3 + 1]; }

private:
    void GetMotion() {
        const auto x = state_->Get(KYN_FIELD_X), q = state_->q(), v = state_->v(), vd = state_->vd();
        auto get = [&](components::Beam& b) {
            for (auto& n : b.nodes) {
                for (int c = 0; c < 7; ++c) {
                    n.position[c] = x[n.id * 7 + c];
                    n.displacement[c] = q[n.id * 7 + c];
                }
                for (int c = 0; c < 6; ++c) {
                    n.velocity[c] = v[n.id * 6 + c];
                    n.acceleration[c] = vd[n.id * 6 + c];
                }
            }
        };
        for (auto& b : turbine_.blades) get(b);
        get(turbine_.tower);
    }

    Context ctx_;
    Model model_;
    components::Turbine turbine_;
    StepParameters parameters_;
    std::unique_ptr<State> state_;
    std::unique_ptr<Elements> elements_;
    std::unique_ptr<Constraints> constraints_;
    std::unique_ptr<Solver> solver_;
    int saved_ = -1;
    std::vector<double> loads_;
};

// src/interfaces/turbine/turbine_interface_builder.hpp
class TurbineInterfaceBuilder {
public:
    components::SolutionBuilder& Solution() { return solution_; }
    components::TurbineBuilder& Turbine() { return turbine_; }
    TurbineInterface Build(const Context& ctx = Context(0)) const {
        return TurbineInterface(ctx, solution_.Input(), turbine_.Input());
    }

private:
    components::SolutionBuilder solution_;
    components::TurbineBuilder turbine_;
};

// ---- CFD interface: floating platform with mooring lines --------------------------
// src/interfaces/cfd/: a platform node with its mass, and per mooring line a
// position-only fairlead rigidly carried by the platform
// (RigidJoint6DOFsTo3DOFs), a position-only anchor (FixedBC3DOFs) and a spring
// between them.  Platform loads in (NodeData::loads -> state.f), motion of every
// node out after each Step(), SaveState / RestoreState and restart files.  The
// model has no beam element and runs as a dense model.
namespace cfd {

using components::NodeData;

// src/interfaces/cfd/mooring_line_input.hpp
struct MooringLineInput {
    double stiffness = 0.;
    double undeformed_length = 0.;
    std::array<double, 3> fairlead_position{0., 0., 0.};
    std::array<double, 3> fairlead_velocity{0., 0., 0.};
    std::array<double, 3> fairlead_acceleration{0., 0., 0.};
    std::array<double, 3> anchor_position{0., 0., 0.};
    std::array<double, 3> anchor_velocity{0., 0., 0.};
    std::array<double, 3> anchor_acceleration{0., 0., 0.};
};

// src/interfaces/cfd/floating_platform_input.hpp
struct FloatingPlatformInput {
    bool enable = false;
    std::array<double, 7> position{0., 0., 0., 1., 0., 0., 0.};
    std::array<double, 6> velocity{0., 0., 0., 0., 0., 0.};
    std::array<double, 6> acceleration{0., 0., 0., 0., 0., 0.};
    std::array<std::array<double, 6>, 6> mass_matrix{};
    std::vector<MooringLineInput> mooring_lines;
};

// src/interfaces/cfd/interface_input.hpp, turbine_input.hpp
struct InterfaceInput {
    std::array<double, 3> gravity{0., 0., 0.};
    double time_step = 0.01;
    double rho_inf = 0.;
    size_t max_iter = 5;
    FloatingPlatformInput floating_platform;
    std::string output_file;
};

// src/interfaces/cfd/mooring_line.hpp, floating_platform.hpp, turbine.hpp
struct MooringLine {
    NodeData fairlead_node;
    NodeData anchor_node;
    size_t fixed_constraint_id;
    size_t rigid_constraint_id;
    size_t spring_element_id;
};
struct FloatingPlatform {
    bool active = false;
    NodeData node{0};
    size_t mass_element_id = 0;
    std::vector<MooringLine> mooring_lines;
};
struct Turbine {
    FloatingPlatform floating_platform;
};

// src/interfaces/cfd/interface.cpp:47-115 (CreateFloatingPlatform)
inline FloatingPlatform CreateFloatingPlatform(const FloatingPlatformInput& in, Model& model) {
    FloatingPlatform p;
    if (!in.enable) return p;
    const auto& x = in.position;
    const auto& v = in.velocity;
    const auto& a = in.acceleration;
    const size_t id = model.AddNode()
                          .SetPosition(x[0], x[1], x[2], x[3], x[4], x[5], x[6])
                          .SetVelocity(v[0], v[1], v[2], v[3], v[4], v[5])
                          .SetAcceleration(a[0], a[1], a[2], a[3], a[4], a[5])
                          .Build();
    p.active = true;
    p.node = NodeData(id);
    p.mass_element_id = model.AddMassElement(id, in.mass_matrix);
    for (const auto& ml : in.mooring_lines) {
        const auto& fp = ml.fairlead_position;
        const auto& fv = ml.fairlead_velocity;
        const auto& fa = ml.fairlead_acceleration;
        const size_t fair = model.AddNode()
                                .SetPosition(fp[0], fp[1], fp[2], 1., 0., 0., 0.)
                                .SetVelocity(fv[0], fv[1], fv[2], 0., 0., 0.)
                                .SetAcceleration(fa[0], fa[1], fa[2], 0., 0., 0.)
                                .Build();
        const auto& ap = ml.anchor_position;
        const auto& av = ml.anchor_velocity;
        const auto& aa = ml.anchor_acceleration;
        const size_t anch = model.AddNode()
                                .SetPosition(ap[0], ap[1], ap[2], 1., 0., 0., 0.)
                                .SetVelocity(av[0], av[1], av[2], 0., 0., 0.)
                                .SetAcceleration(aa[0], aa[1], aa[2], 0., 0., 0.)
                                .Build();
        const size_t fixed = model.AddFixedBC3DOFs(anch);
        const size_t rigid = model.AddRigidJoint6DOFsTo3DOFs({id, fair});
        const size_t spring = model.AddSpringElement(fair, anch, ml.stiffness, ml.undeformed_length);
        p.mooring_lines.push_back({NodeData(fair), NodeData(anch), fixed, rigid, spring});
    }
    return p;
}

// src/interfaces/cfd/interface.hpp
class Interface {
public:
    Interface(const Context& ctx, const InterfaceInput& in)
        : ctx_(ctx), model_(in.gravity), parameters_(true, in.max_iter, in.time_step, in.rho_inf) {
        turbine.floating_platform = CreateFloatingPlatform(in.floating_platform, model_);
        auto [state, elements, constraints, solver] = model_.CreateSystemWithSolver(ctx_);
        state_ = std::make_unique<State>(state);
        elements_ = std::make_unique<Elements>(elements);
        constraints_ = std::make_unique<Constraints>(constraints);
        solver_ = std::make_unique<Solver>(solver);
        saved_ = kyn_model_clone(ctx_.get(), solver_->model()->id);  // state_save (CloneState)
        check(ctx_.get(), saved_);
        loads_.assign(solver_->model()->info.num_nodes * 6, 0.);
        GetMotion();
    }
    Interface(const Interface&) = delete;
    Interface& operator=(const Interface&) = delete;
    Interface(Interface&& o) noexcept
        : turbine(std::move(o.turbine)), ctx_(o.ctx_), model_(std::move(o.model_)), parameters_(o.parameters_),
          state_(std::move(o.state_)), elements_(std::move(o.elements_)), constraints_(std::move(o.constraints_)),
          solver_(std::move(o.solver_)), saved_(o.saved_), loads_(std::move(o.loads_)) {
        o.saved_ = -1;
    }
    ~Interface() {
        if (saved_ >= 0) kyn_model_destroy(ctx_.get(), saved_);
    }

    Turbine turbine;

    // Platform loads -> state.f, one step, motion back (interface.cpp:270-296).
    bool Step() {
        const auto& p = turbine.floating_platform;
        if (p.active)
            for (int c = 0; c < 6; ++c) loads_[p.node.id * 6 + c] = p.node.loads[c];
        state_->SetExternalForces(loads_);
        if (!kynema_b200::Step(parameters_, *solver_, *elements_, *state_, *constraints_)) return false;
        GetMotion();
        return true;
    }
    void SaveState() { check(ctx_.get(), kyn_state_copy(ctx_.get(), saved_, solver_->model()->id)); }
    void RestoreState() {
        check(ctx_.get(), kyn_state_copy(ctx_.get(), solver_->model()->id, saved_));
        GetMotion();
    }
    // WriteStateToFile / ReadStateFromFile records (interface.cpp:249-262)
    void WriteRestart(const std::string& filename) const {
        size_t bytes = 0;
        check(ctx_.get(), kyn_state_write(ctx_.get(), solver_->model()->id, nullptr, 0, &bytes));
        std::vector<char> buf(bytes);
        check(ctx_.get(), kyn_state_write(ctx_.get(), solver_->model()->id, buf.data(), buf.size(), &bytes));
        FILE* f = std::fopen(filename.c_str(), "wb");
        if (!f) throw std::runtime_error("cannot open restart file for writing: " + filename);
        const size_t w = std::fwrite(buf.data(), 1, buf.size(), f);
        std::fclose(f);
        if (w != buf.size()) throw std::runtime_error("short write of restart file: " + filename);
    }
    void ReadRestart(const std::string& filename) {
        FILE* f = std::fopen(filename.c_str(), "rb");
        if (!f) throw std::runtime_error("cannot open restart file: " + filename);
        std::vector<char> buf;
        char chunk[4096];
        size_t r = 0;
        while ((r = std::fread(chunk, 1, sizeof(chunk), f)) > 0) buf.insert(buf.end(), chunk, chunk + r);
        std::fclose(f);
        check(ctx_.get(), kyn_state_read(ctx_.get(), solver_->model()->id, buf.data(), buf.size()));
        GetMotion();
    }

private:
    void GetMotion() {
        auto& p = turbine.floating_platform;
        if (!p.active) return;
        const auto x = state_->Get(KYN_FIELD_X), q = state_->q(), v = state_->v(), vd = state_->vd();
        auto fill = [&](NodeData& n) {
            for (int c = 0; c < 7; ++c) {
                n.position[c] = x[n.id * 7 + c];
                n.displacement[c] = q[n.id * 7 + c];
            }
            for (int c = 0; c < 6; ++c) {
                n.velocity[c] = v[n.id * 6 + c];
                n.acceleration[c] = vd[n.id * 6 + c];
            }
        };
        fill(p.node);
        for (auto& ml : p.mooring_lines) {
            fill(ml.fairlead_node);
            fill(ml.anchor_node);
        }
    }

    Context ctx_;
    Model model_;
    StepParameters parameters_;
    std::unique_ptr<State> state_;
    std::unique_ptr<Elements> elements_;
    std::unique_ptr<Constraints> constraints_;
    std::unique_ptr<Solver> solver_;
    int saved_ = -1;
    std::vector<double> loads_;
};

// src/interfaces/cfd/interface_builder.hpp
class InterfaceBuilder {
public:
    InterfaceBuilder& SetGravity(const std::array<double, 3>& g) { in_.gravity = g; return *this; }
    InterfaceBuilder& SetTimeStep(double h) { in_.time_step = h; return *this; }
    InterfaceBuilder& SetDampingFactor(double rho) { in_.rho_inf = rho; return *this; }
    InterfaceBuilder& SetMaximumNonlinearIterations(size_t n) { in_.max_iter = n; return *this; }
    InterfaceBuilder& EnableFloatingPlatform(bool on) { in_.floating_platform.enable = on; return *this; }
    InterfaceBuilder& SetFloatingPlatformPosition(const std::array<double, 7>& p) {
        in_.floating_platform.position = p;
        return *this;
    }
    InterfaceBuilder& SetFloatingPlatformVelocity(const std::array<double, 6>& v) {
        in_.floating_platform.velocity = v;
        return *this;
    }
    InterfaceBuilder& SetFloatingPlatformAcceleration(const std::array<double, 6>& a) {
        in_.floating_platform.acceleration = a;
        return *this;
    }
    InterfaceBuilder& SetFloatingPlatformMassMatrix(const std::array<std::array<double, 6>, 6>& m) {
        in_.floating_platform.mass_matrix = m;
        return *this;
    }
    InterfaceBuilder& SetNumberOfMooringLines(size_t n) {
        in_.floating_platform.mooring_lines.resize(n);
        return *this;
    }
    InterfaceBuilder& SetMooringLineStiffness(size_t i, double k) { line(i).stiffness = k; return *this; }
    InterfaceBuilder& SetMooringLineUndeformedLength(size_t i, double l) {
        line(i).undeformed_length = l;
        return *this;
    }
    InterfaceBuilder& SetMooringLineFairleadPosition(size_t i, const std::array<double, 3>& p) {
        line(i).fairlead_position = p;
        return *this;
    }
    InterfaceBuilder& SetMooringLineAnchorPosition(size_t i, const std::array<double, 3>& p) {
        line(i).anchor_position = p;
        return *this;
    }
    // NetCDF output is not part of this path; the path is recorded only
    InterfaceBuilder& SetOutputFile(const std::string& f) { in_.output_file = f; return *this; }
    Interface Build(const Context& ctx = Context(0)) const { return Interface(ctx, in_); }

private:
    MooringLineInput& line(size_t i) {
        if (i >= in_.floating_platform.mooring_lines.size())
            throw std::out_of_range("mooring line index beyond SetNumberOfMooringLines");
        return in_.floating_platform.mooring_lines[i];
    }
    InterfaceInput in_;
};

}  // namespace cfd

}  // namespace kynema_b200::interfaces
