// The reference's regression drivers written against the C++ shim (kynema_b200.hpp):
// test_cantilever_beam.cpp:31-138, test_rotating_beam.cpp:93-150, :390-456
// (rotation control) and :581-680 (generator torque on a revolute joint),
// test_spring_mass_system.cpp:23-96, test_heavy_top.cpp:9-75, same inputs, same golden
// tolerances.  Exit code 0 on success.
#include <cmath>
#include <cstdio>
#include <vector>

#include "kynema_b200.hpp"

using namespace kynema_b200;

static int failures = 0;
static void expect_near(double a, double b, double tol, const char* what) {
    if (!(std::abs(a - b) <= tol)) {
        std::printf("FAIL %s: %.17g vs %.17g\n", what, a, b);
        ++failures;
    }
}

constexpr std::array<std::array<double, 6>, 6> kMass = {{
    {8.538e-2, 0., 0., 0., 0., 0.}, {0., 8.538e-2, 0., 0., 0., 0.}, {0., 0., 8.538e-2, 0., 0., 0.},
    {0., 0., 0., 1.4433e-2, 0., 0.}, {0., 0., 0., 0., 0.40972e-2, 0.}, {0., 0., 0., 0., 0., 1.0336e-2}}};
constexpr std::array<std::array<double, 6>, 6> kStiff = {{
    {1368.17e3, 0., 0., 0., 0., 0.}, {0., 88.56e3, 0., 0., 0., 0.}, {0., 0., 38.78e3, 0., 0., 0.},
    {0., 0., 0., 16.9600e3, 17.6100e3, -0.3510e3}, {0., 0., 0., 17.6100e3, 59.1200e3, -0.3700e3},
    {0., 0., 0., -0.3510e3, -0.3700e3, 141.470e3}}};
const std::vector<std::array<double, 2>> kGauss7 = {
    {-0.9491079123427585, 0.1294849661688697}, {-0.7415311855993943, 0.27970539148927664},
    {-0.40584515137739696, 0.3818300505051189}, {6.123233995736766e-17, 0.4179591836734694},
    {0.4058451513773971, 0.3818300505051189}, {0.7415311855993945, 0.27970539148927664},
    {0.9491079123427585, 0.1294849661688697}};

static void cantilever(const Context& ctx) {
    const std::vector<double> node_s{0., 0.17267316464601146, 0.5, 0.8273268353539885, 1.};
    Model model;
    model.SetGravity(0., 0., 0.);
    std::vector<size_t> ids;
    for (double s : node_s) ids.push_back(model.AddNode().SetElemLocation(s).SetPosition(10 * s, 0., 0., 1., 0., 0., 0.).Build());
    const std::vector<BeamSection> sections{BeamSection(0., kMass, kStiff), BeamSection(1., kMass, kStiff)};
    model.AddBeamElement(ids, sections, kGauss7);
    model.AddFixedBC(ids[0]);
    auto parameters = StepParameters(true, 5, 0.005, 0.0);
    auto [state, elements, constraints, solver] = model.CreateSystemWithSolver(ctx);
    const double expected[3][3] = {{-8.15173937E-08, -1.86549248E-07, 6.97278045E-04},
                                   {-1.00926258E-06, -7.91711079E-07, 2.65017558E-03},
                                   {-5.05830945E-06, -2.29457246E-06, 6.30508154E-03}};
    for (int k = 0; k < 3; ++k) {
        elements.SetNodeFX(0, ids.back(), 2, 100. * std::sin(10.0 * 0.005 * (k + 1)));
        const bool converged = Step(parameters, solver, elements, state, constraints);
        if (!converged) { std::printf("FAIL cantilever step %d not converged\n", k); ++failures; }
        const auto q = state.q();
        for (int c = 0; c < 3; ++c) expect_near(q[4 * 7 + c], expected[k][c], 1e-6, "cantilever tip q");
    }
}

static void rotating_beam(const Context& ctx) {
    const std::vector<double> node_s{0., 0.11747233803526763, 0.35738424175967748, 0.64261575824032247, 0.88252766196473242, 1.};
    Model model;
    model.SetGravity(0., 0., 0.);
    std::vector<size_t> ids;
    for (double s : node_s) ids.push_back(model.AddNode().SetElemLocation(s).SetPosition(10 * s, 0., 0., 1., 0., 0., 0.).Build());
    const std::vector<BeamSection> sections{BeamSection(0., kMass, kStiff), BeamSection(1., kMass, kStiff)};
    model.AddBeamElement(ids, sections, kGauss7);
    model.TranslateBeam(0, {2., 0., 0.});
    model.SetBeamVelocityAboutPoint(0, {0., 0., 0., 0., 0., 0.1}, {0., 0., 0.});
    model.AddPrescribedBC(ids[0]);
    auto [state, elements, constraints, solver] = model.CreateSystemWithSolver(ctx);
    auto parameters = StepParameters(true, 5, 0.01, 0.9);
    for (int i = 0; i < 10; ++i) {
        const auto q = RotationVectorToQuaternion({0., 0., 0.1 * 0.01 * (i + 1)});
        const auto xr = RotateVectorByQuaternion(q, {2., 0., 0.});
        constraints.UpdateDisplacement(0, {xr[0] - 2., xr[1], xr[2], q[0], q[1], q[2], q[3]});
        if (!Step(parameters, solver, elements, state, constraints)) { std::printf("FAIL rotating step %d\n", i); ++failures; }
    }
    // first row of the golden q (test_rotating_beam.cpp:142-150)
    const auto q = state.q();
    const double root[7] = {-0.000099999166669473282, 0.019999666668333329, 0., 0.99998750002604219, 0., 0., 0.0049999791666927116};
    for (int c = 0; c < 7; ++c) expect_near(q[c], root[c], 1e-6, "rotating beam root q");
    if (solver.convergence_err().empty()) { std::printf("FAIL empty convergence history\n"); ++failures; }
}

// test_rotating_beam.cpp:390-456: pitch through a control signal the shim reads before each Step
static void rotation_control(const Context& ctx) {
    const std::vector<double> node_s{0., 0.11747233803526763, 0.35738424175967748, 0.64261575824032247, 0.88252766196473242, 1.};
    Model model;
    model.SetGravity(0., 0., 0.);
    std::vector<size_t> ids;
    for (double s : node_s) ids.push_back(model.AddNode().SetElemLocation(s).SetPosition(10 * s, 0., 0., 1., 0., 0., 0.).Build());
    const std::vector<BeamSection> sections{BeamSection(0., kMass, kStiff), BeamSection(1., kMass, kStiff)};
    model.AddBeamElement(ids, sections, kGauss7);
    model.TranslateBeam(0, {2., 0., 0.});
    double pitch = 0.;
    const size_t hub = model.AddNode().SetPosition(0., 0., 0., 1., 0., 0., 0.).Build();
    model.AddRotationControl({hub, ids.front()}, {1., 0., 0.}, &pitch);
    model.AddFixedBC(hub);
    auto [state, elements, constraints, solver] = model.CreateSystemWithSolver(ctx);
    auto parameters = StepParameters(true, 5, 0.01, 0.9);
    for (int i = 0; i < 10; ++i) {
        pitch = 0.01 * (i + 1) * 3.14159265358979323846 / 2.;
        if (!Step(parameters, solver, elements, state, constraints)) { std::printf("FAIL rotation control step %d\n", i); ++failures; }
    }
    // rows 0 and 5 of the golden q (test_rotating_beam.cpp:436-456)
    const auto q = state.q();
    const double root[7] = {-5.7690945215728628E-18, 2.0652319043893875E-18, -2.4953577261422928E-20,
                            0.99691733356165013, 0.078459097906677058, 5.0946025505270351E-19, 3.3980589449407732E-19};
    const double tip[7] = {-0.0000058187577280119813, -0.00014174393267219577, 0.0015608892113182621,
                           0.9972883429355086, 0.073590276246437658, -0.00065565396382017294, -0.000049038763777556399};
    for (int c = 0; c < 7; ++c) expect_near(q[c], root[c], 1e-6, "rotation control root q");
    for (int c = 0; c < 7; ++c) expect_near(q[5 * 7 + c], tip[c], 1e-6, "rotation control tip q");
}

// test_rotating_beam.cpp:581-680 (GeneratorTorqueWithAxisTilt): shaft base (fixed) ->
// revolute joint about the tilted shaft -> azimuth -> rigid -> hub -> rigid -> blade
// root, generator torque read through the pointer before each Step; azimuth q, v and
// the joint output after 10 steps at the test's 1e-6
static void generator_torque(const Context& ctx, double tilt, const double (&az_q)[7],
                             const double (&az_v)[6], const double (&out)[3]) {
    const std::vector<double> node_s{0., 0.11747233803526763, 0.35738424175967748, 0.64261575824032247, 0.88252766196473242, 1.};
    Model model;
    model.SetGravity(0., 0., 0.);
    std::vector<size_t> ids;
    for (double s : node_s) ids.push_back(model.AddNode().SetElemLocation(s).SetPosition(10 * s, 0., 0., 1., 0., 0., 0.).Build());
    const std::vector<BeamSection> sections{BeamSection(0., kMass, kStiff), BeamSection(1., kMass, kStiff)};
    model.AddBeamElement(ids, sections, kGauss7);
    model.TranslateBeam(0, {2., 0., 0.});
    model.RotateBeamAboutPoint(0, RotationVectorToQuaternion({tilt, 0., 0.}), {0., 0., 0.});
    const size_t shaft = model.AddNode().SetPosition(0., 0., 0., 1., 0., 0., 0.).Build();
    const size_t azimuth = model.AddNode().SetPosition(0., 0., 0., 1., 0., 0., 0.).Build();
    const size_t hub = model.AddNode().SetPosition(0., std::sin(tilt), std::cos(tilt), 1., 0., 0., 0.).Build();
    model.AddFixedBC(shaft);
    double torque = 100.;
    const size_t rj = model.AddRevoluteJointConstraint({shaft, azimuth}, {0., std::sin(tilt), std::cos(tilt)}, &torque);
    model.AddRigidJointConstraint({azimuth, hub});
    model.AddRigidJointConstraint({hub, ids.front()});
    auto [state, elements, constraints, solver] = model.CreateSystemWithSolver(ctx);
    auto parameters = StepParameters(true, 5, 0.01, 0.);
    for (int i = 0; i < 10; ++i)
        if (!Step(parameters, solver, elements, state, constraints)) { std::printf("FAIL generator torque step %d\n", i); ++failures; }
    const auto q = state.q();
    const auto v = state.v();
    const auto o = constraints.output();
    for (int c = 0; c < 7; ++c) expect_near(q[azimuth * 7 + c], az_q[c], 1e-6, "generator torque azimuth q");
    for (int c = 0; c < 6; ++c) expect_near(v[azimuth * 6 + c], az_v[c], 1e-6, "generator torque azimuth v");
    for (int c = 0; c < 3; ++c) expect_near(o[rj * 3 + c], out[c], 1e-6, "generator torque joint output");
}

// test_heavy_top.cpp:9-75: a top held at a point (RigidJoint6DOFsTo3DOFs to a
// position-only ground node with PrescribedBC3DOFs), q after 400 steps at 1e-10
static void heavy_top(const Context& ctx) {
    Model model;
    model.SetGravity(0., 0., -9.81);
    const double omega[3] = {0., 150., -4.61538};
    const double x[3] = {0., 1., 0.};
    const double xd[3] = {omega[1] * x[2] - omega[2] * x[1], omega[2] * x[0] - omega[0] * x[2],
                          omega[0] * x[1] - omega[1] * x[0]};
    const size_t top = model.AddNode()
                           .SetPosition(x[0], x[1], x[2], 1., 0., 0., 0.)
                           .SetVelocity(xd[0], xd[1], xd[2], omega[0], omega[1], omega[2])
                           .SetAcceleration(0., -21.3017325444000001, -30.9608307692308244, 661.3461692307691919, 0., 0.)
                           .Build();
    model.AddMassElement(top, {{{15., 0., 0., 0., 0., 0.}, {0., 15., 0., 0., 0., 0.}, {0., 0., 15., 0., 0., 0.},
                                {0., 0., 0., 0.234375, 0., 0.}, {0., 0., 0., 0., 0.46875, 0.}, {0., 0., 0., 0., 0., 0.234375}}});
    const size_t ground = model.AddNode().SetPosition(0., 0., 0., 1., 0., 0., 0.).Build();
    model.AddRigidJoint6DOFsTo3DOFs({top, ground});
    model.AddPrescribedBC3DOFs(ground);
    auto parameters = StepParameters(true, 10, 0.002, 0.9, 1e-5, 1e-3);
    auto [state, elements, constraints, solver] = model.CreateSystemWithSolver(ctx);
    for (int i = 0; i < 400; ++i)
        if (!Step(parameters, solver, elements, state, constraints)) { std::printf("FAIL heavy top step %d\n", i); ++failures; }
    const double expect[7] = {-0.42217802273894345, -0.09458263530050703, -0.04455460488952848, -0.17919607435565366,
                              0.21677896640311572, -0.9594776960853596, -0.017268392381761217};
    const auto q = state.q();
    for (int c = 0; c < 7; ++c) expect_near(q[c], expect[c], 1e-10, "heavy top q");
}

// test_spring_mass_system.cpp:23-96: a mass on a spring to a fixed node, no beam element
static void spring_mass(const Context& ctx) {
    Model model;
    const size_t fixed = model.AddNode().SetPosition(0., 0., 0., 1., 0., 0., 0.).Build();
    const size_t mass = model.AddNode().SetPosition(2., 0., 0., 1., 0., 0., 0.).Build();
    model.AddMassElement(mass, {{{1., 0., 0., 0., 0., 0.}, {0., 1., 0., 0., 0., 0.}, {0., 0., 1., 0., 0., 0.},
                                 {0., 0., 0., 1., 0., 0.}, {0., 0., 0., 0., 1., 0.}, {0., 0., 0., 0., 0., 1.}}});
    model.AddFixedBC(fixed);
    model.AddSpringElement(fixed, mass, 10., 0.);
    const double T = 2. * 3.14159265358979323846 * std::sqrt(1. / 10.);
    auto parameters = StepParameters(true, 6, T / 1000., 0.);
    auto [state, elements, constraints, solver] = model.CreateSystemWithSolver(ctx);
    for (int i = 1; i <= 1000; ++i) {
        if (!Step(parameters, solver, elements, state, constraints)) { std::printf("FAIL spring-mass step %d\n", i); ++failures; }
        if (i == 500) expect_near(state.q()[7], -3.9999199193098396, 1e-12, "spring-mass x at T/2");
    }
    expect_near(state.q()[7], -8.1226588438437419e-05, 1e-12, "spring-mass x at T");
}

int main() {
    try {
        Context ctx(0);
        cantilever(ctx);
        rotating_beam(ctx);
        rotation_control(ctx);
        generator_torque(ctx, 0., {0., 0., 0., 0.99998634, 0., 0., -0.0052267}, {0., 0., 0., 0., 0., -0.18978539},
                         {-0.01045353, -0.18978539, -0.566558});
        generator_torque(ctx, 3.14159265358979323846 / 2., {0., 0., 0., 0.99998634, 0., -0.0052267, 0.},
                         {0., 0., 0., 0., -0.18978539, 0.}, {-0.01045353, -0.18978539, -0.566560});
        spring_mass(ctx);
        heavy_top(ctx);
    } catch (const std::exception& e) {
        std::printf("FAIL exception: %s\n", e.what());
        return 2;
    }
    std::printf("%s (%d failures)\n", failures ? "FAILED" : "OK", failures);
    return failures ? 1 : 0;
}
