// The reference's blade-interface regression drivers written against
// kynema_b200_interfaces.hpp: BladeInterfaceTest.RotatingBeam,
// BladeInterfaceTest.BladeWindIO and BladeInterfaceTest.StaticCurledBeam
// (tests/regression_tests/interfaces/test_blade_interface.cpp:13-277, 392-492),
// same inputs, same golden values and tolerances (1e-10; 1e-8 static).  The IEA-15 blade input of
// the WindIO case is read from the fixture given as argv[1]
// (tests/golden/iea15_blade_windio.txt).  Exit code 0 on success.
#include <cmath>
#include <cstdio>
#include <fstream>
#include <numbers>
#include <sstream>
#include <string>
#include <vector>

#include "kynema_b200_interfaces.hpp"

using namespace kynema_b200;
using namespace kynema_b200::interfaces;

static int failures = 0;
static void expect_near(double a, double b, double tol, const char* what, int i) {
    if (!(std::abs(a - b) <= tol)) {
        std::printf("FAIL %s[%d]: %.17g vs %.17g\n", what, i, a, b);
        ++failures;
    }
}

// BladeWindIO: an 11-node IEA-15 blade described along z (WindIO), twisted,
// with 26 sections; an oscillating moment at the tip for 19 steps.
static void blade_windio(const char* path) {
    std::ifstream in(path);
    if (!in) throw std::runtime_error(std::string("cannot open ") + path);
    std::string line, text;
    while (std::getline(in, line))
        if (line.empty() || line[0] != '#') text += line + "\n";
    std::istringstream f(text);
    BladeInterfaceBuilder builder;
    builder.Solution()
        .EnableDynamicSolve()
        .SetTimeStep(0.01)
        .SetDampingFactor(0.0)
        .SetMaximumNonlinearIterations(6)
        .SetAbsoluteErrorTolerance(1e-6)
        .SetRelativeErrorTolerance(1e-4);
    builder.Blade().SetElementOrder(10).PrescribedRootMotion(true);
    const auto Z = components::ReferenceAxisOrientation::Z;
    size_t n = 0;
    f >> n;
    for (size_t i = 0; i < n; ++i) {
        double g, x, y, z;
        f >> g >> x >> y >> z;
        builder.Blade().AddRefAxisPoint(g, {x, y, z}, Z);
    }
    f >> n;
    for (size_t i = 0; i < n; ++i) {
        double g, t;
        f >> g >> t;
        builder.Blade().AddRefAxisTwist(g, t * std::numbers::pi / 180.);
    }
    f >> n;
    for (size_t i = 0; i < n; ++i) {
        double g, m[21], k[21];
        f >> g;
        for (double& v : m) f >> v;
        for (double& v : k) f >> v;
        auto full = [](const double* a) {
            return std::array<std::array<double, 6>, 6>{{{a[0], a[1], a[2], a[3], a[4], a[5]},
                                                          {a[1], a[6], a[7], a[8], a[9], a[10]},
                                                          {a[2], a[7], a[11], a[12], a[13], a[14]},
                                                          {a[3], a[8], a[12], a[15], a[16], a[17]},
                                                          {a[4], a[9], a[13], a[16], a[18], a[19]},
                                                          {a[5], a[10], a[14], a[17], a[19], a[20]}}};
        };
        builder.Blade().AddSection(g, full(m), full(k), Z);
    }
    double expected[7];
    for (double& v : expected) f >> v;
    if (!f) throw std::runtime_error("truncated WindIO fixture");
    auto interface = builder.Build(Context(0));
    auto& tip = interface.Blade().nodes.back();
    for (int i = 1; i < 20; ++i) {
        const double t = static_cast<double>(i) * 0.01;
        tip.loads[1] = 2.0e5 * std::sin(2. * std::numbers::pi * 0.05 * t);
        if (!interface.Step()) {
            std::printf("FAIL windio step %d did not converge\n", i);
            ++failures;
            return;
        }
    }
    for (int c = 0; c < 7; ++c) expect_near(tip.position[c], expected[c], 1e-10, "windio tip position", c);
}

// StaticCurledBeam: static solves of a straight 10 m blade of order 10 (two key
// points, sections refined once) under a growing tip moment about y that curls
// it towards a full circle; tip position after each load at 1e-8.
static void static_curled_beam() {
    BladeInterfaceBuilder builder;
    builder.Solution()
        .EnableStaticSolve()
        .SetTimeStep(1.)
        .SetDampingFactor(1.)
        .SetMaximumNonlinearIterations(10)
        .SetAbsoluteErrorTolerance(1e-5)
        .SetRelativeErrorTolerance(1e-3);
    builder.Blade().SetElementOrder(10).SetSectionRefinement(1).PrescribedRootMotion(true)
        .AddRefAxisTwist(0., 0.).AddRefAxisTwist(1., 0.);
    const auto X = components::ReferenceAxisOrientation::X;
    for (double s : {0., 1.}) builder.Blade().AddRefAxisPoint(s, {s * 10., 0., 0.}, X);
    for (int i = 0; i <= 10; ++i)
        builder.Blade().AddSection(
            0.1 * i,
            {{{1., 0., 0., 0., 0., 0.}, {0., 1., 0., 0., 0., 0.}, {0., 0., 1., 0., 0., 0.},
              {0., 0., 0., 1., 0., 0.}, {0., 0., 0., 0., 1., 0.}, {0., 0., 0., 0., 0., 1.}}},
            {{{1770.e3, 0., 0., 0., 0., 0.}, {0., 1770.e3, 0., 0., 0., 0.}, {0., 0., 1770.e3, 0., 0., 0.},
              {0., 0., 0., 8.16e3, 0., 0.}, {0., 0., 0., 0., 86.9e3, 0.}, {0., 0., 0., 0., 0., 215.e3}}},
            X);
    auto interface = builder.Build(Context(0));
    auto& tip = interface.Blade().nodes.back();
    const double moments[6] = {0., 10920.0, 21840.0, 32761.0, 43681.0, 54601.0};
    const double expected[6][3] = {{10., 0., 0.},
                                   {7.5396813678794645, 0., 5.5363879677563252},
                                   {2.275087482106132, 0., 7.2166560706481686},
                                   {-1.6222827675944771, 0., 4.7694966546892239},
                                   {-1.9054629771623546, 0., 1.3243726828814482},
                                   {0.021386893541979646, 0., 0.0006097054603659835}};
    for (int k = 0; k < 6; ++k) {
        tip.loads[4] = -moments[k];
        if (!interface.Step()) {
            std::printf("FAIL static curled beam load %d did not converge\n", k);
            ++failures;
            return;
        }
        for (int c = 0; c < 3; ++c) expect_near(tip.position[c], expected[k][c], 1e-8, "curled tip", 3 * k + c);
    }
}

// TwoBeams (test_blade_interface.cpp:312-372): two order-3 beams built by
// BeamBuilder from a straight axis, the second moved 10 m along x, a
// PrescribedBC at the first root and a RigidJoint from the first tip to the
// second root (one dense bordered system); every one of 1000 steps converges.
static void two_beams() {
    components::BeamBuilder builder;
    const int n_nodes = 4;
    builder.SetElementOrder(n_nodes - 1).PrescribedRootMotion(false)
        .SetRootPosition({0., 0., 0., 1., 0., 0., 0.}).AddRefAxisTwist(0., 0.).AddRefAxisTwist(1., 0.);
    const int n_kps = 12;
    for (int i = 0; i < n_kps; ++i) {
        const double s = static_cast<double>(i) / (n_kps - 1);
        builder.AddRefAxisPoint(s, {10. * s, 0., 0.}, components::ReferenceAxisOrientation::X);
    }
    for (int i = 0; i <= 20; ++i)
        builder.AddSection(
            0.05 * i,
            {{{8.538e-2, 0., 0., 0., 0., 0.}, {0., 8.538e-2, 0., 0., 0., 0.}, {0., 0., 8.538e-2, 0., 0., 0.},
              {0., 0., 0., 1.4433e-2, 0., 0.}, {0., 0., 0., 0., 0.40972e-2, 0.}, {0., 0., 0., 0., 0., 1.0336e-2}}},
            {{{1368.17e3, 0., 0., 0., 0., 0.}, {0., 88.56e3, 0., 0., 0., 0.}, {0., 0., 38.78e3, 0., 0., 0.},
              {0., 0., 0., 16.9600e3, 17.6100e3, -0.3510e3}, {0., 0., 0., 17.6100e3, 59.1200e3, -0.3700e3},
              {0., 0., 0., -0.3510e3, -0.3700e3, 141.470e3}}},
            components::ReferenceAxisOrientation::X);
    Model model({0., 0., -9.81});
    components::Beam beam_1(builder.Input(), model);
    components::Beam beam_2(builder.Input(), model);
    for (auto& node : beam_2.nodes) model.GetNode(node.id).x0[0] += 10.;
    model.AddPrescribedBC(beam_1.nodes[0].id);
    model.AddRigidJointConstraint({beam_1.nodes[n_nodes - 1].id, beam_2.nodes[0].id});
    const StepParameters parameters(true, 6, 0.01, 0.);
    auto [state, elements, constraints, solver] = model.CreateSystemWithSolver(Context(0));
    for (int i = 0; i < 1000; ++i)
        if (!Step(parameters, solver, elements, state, constraints)) {
            std::printf("FAIL two beams: step %d did not converge\n", i);
            ++failures;
            return;
        }
}

int main(int argc, char** argv) {
    try {
        if (argc > 1) blade_windio(argv[1]);
        static_curled_beam();
        two_beams();
        const double time_step = 0.01;
        const std::array<double, 3> omega{0., 0., 1.};
        const std::array<double, 3> x0_root{2., 0., 0.};
        const std::array<double, 3> root_vel{omega[1] * x0_root[2] - omega[2] * x0_root[1],
                                             omega[2] * x0_root[0] - omega[0] * x0_root[2],
                                             omega[0] * x0_root[1] - omega[1] * x0_root[0]};
        BladeInterfaceBuilder builder;
        builder.Solution()
            .EnableDynamicSolve()
            .SetTimeStep(time_step)
            .SetDampingFactor(0.0)
            .SetMaximumNonlinearIterations(6)
            .SetAbsoluteErrorTolerance(1e-6)
            .SetRelativeErrorTolerance(1e-4);
        const std::vector<double> node_s{0., 0.11747233803526763, 0.35738424175967748,
                                         0.64261575824032247, 0.88252766196473242, 1.};
        builder.Blade()
            .SetElementOrder(5)
            .PrescribedRootMotion(true)
            .SetRootPosition({x0_root[0], x0_root[1], x0_root[2], 1., 0., 0., 0.})
            .SetRootVelocity({root_vel[0], root_vel[1], root_vel[2], omega[0], omega[1], omega[2]})
            .AddRefAxisTwist(0., 0.)
            .AddRefAxisTwist(1., 0.);
        for (double s : node_s)
            builder.Blade().AddRefAxisPoint(s, {10. * s, 0., 0.}, components::ReferenceAxisOrientation::X);
        const std::vector<double> section_s{0.0254460438286208, 0.1292344072003028, 0.2970774243113015, 0.5,
                                            0.7029225756886985, 0.8707655927996972, 0.9745539561713792};
        const components::ReferenceAxisOrientation X = components::ReferenceAxisOrientation::X;
        for (double s : section_s)
            builder.Blade().AddSection(
                s,
                {{{8.538e-2, 0., 0., 0., 0., 0.}, {0., 8.538e-2, 0., 0., 0., 0.}, {0., 0., 8.538e-2, 0., 0., 0.},
                  {0., 0., 0., 1.4433e-2, 0., 0.}, {0., 0., 0., 0., 0.40972e-2, 0.}, {0., 0., 0., 0., 0., 1.0336e-2}}},
                {{{1368.17e3, 0., 0., 0., 0., 0.}, {0., 88.56e3, 0., 0., 0., 0.}, {0., 0., 38.78e3, 0., 0., 0.},
                  {0., 0., 0., 16.9600e3, 17.6100e3, -0.3510e3}, {0., 0., 0., 17.6100e3, 59.1200e3, -0.3700e3},
                  {0., 0., 0., -0.3510e3, -0.3700e3, 141.470e3}}},
                X);
        auto interface = builder.Build(Context(0));
        for (int i = 1; i < 10; ++i) {
            const double t = static_cast<double>(i) * time_step;
            const auto u_rot = RotationVectorToQuaternion({omega[0] * t, omega[1] * t, omega[2] * t});
            const auto x_root = RotateVectorByQuaternion(u_rot, x0_root);
            interface.SetRootDisplacement({x_root[0] - x0_root[0], x_root[1] - x0_root[1], x_root[2] - x0_root[2],
                                           u_rot[0], u_rot[1], u_rot[2], u_rot[3]});
            if (!interface.Step()) {
                std::printf("FAIL step %d did not converge\n", i);
                ++failures;
            }
        }
        const auto& root = interface.Blade().nodes[0];
        const auto& tip = interface.Blade().nodes[5];
        const double rp[7] = {1.9919054660239885, 0.17975709839602211, 0., 0.99898767084784234, 0., 0.,
                              0.044984814037660227};
        const double ru[7] = {-0.0080945339760114532, 0.17975709839602211, 0., 0.99898767084784234, 0., 0.,
                              0.044984814037660227};
        const double rv[6] = {-0.17976259212149071, 1.9919719054875213, 0., 0., 0., 1.};
        const double ra[6] = {-1.9920882238788629, -0.17977158309645525, 0., 0., 0., 0.};
        const double tp[7] = {11.951460424343411, 1.0785463019560009, 2.2845605555050727E-10, 0.99898766738195299,
                              2.6570959740959799E-9, -1.0123941616837804E-10, 0.044984891005365443};
        const double tu[7] = {-0.048539575656588806, 1.0785463019560009, 2.2845605555050727E-10,
                              0.99898766738195299, 2.6570959740959799E-9, -1.0123941616837804E-10,
                              0.044984891005365443};
        const double tv[6] = {-1.0786835619583102, 11.95303967174639, -6.3862048021175104E-8,
                              0.000003159329892760129, 2.5866107917084571E-7, 1.0001562024381443};
        const double ta[6] = {-11.955952417551353, -1.0800839943831992, -0.000013544534439173783,
                              -0.000046709402446003812, 0.000008256203749646939, 0.00020635762959181575};
        for (int c = 0; c < 7; ++c) {
            expect_near(root.position[c], rp[c], 1e-10, "root position", c);
            expect_near(root.displacement[c], ru[c], 1e-10, "root displacement", c);
            expect_near(tip.position[c], tp[c], 1e-10, "tip position", c);
            expect_near(tip.displacement[c], tu[c], 1e-10, "tip displacement", c);
        }
        for (int c = 0; c < 6; ++c) {
            expect_near(root.velocity[c], rv[c], 1e-10, "root velocity", c);
            expect_near(root.acceleration[c], ra[c], 1e-10, "root acceleration", c);
            expect_near(tip.velocity[c], tv[c], 1e-10, "tip velocity", c);
            expect_near(tip.acceleration[c], ta[c], 1e-10, "tip acceleration", c);
        }
        // save / restore: a step taken after SaveState is undone by RestoreState
        interface.SaveState();
        const auto before = tip.position;
        interface.Blade().nodes[5].loads[2] = 1e3;
        interface.Step();
        interface.RestoreState();
        for (int c = 0; c < 7; ++c) expect_near(interface.Blade().nodes[5].position[c], before[c], 0., "restored", c);
    } catch (const std::exception& e) {
        std::printf("FAIL exception: %s\n", e.what());
        return 2;
    }
    std::printf("%s (%d failures)\n", failures ? "FAILED" : "OK", failures);
    return failures ? 1 : 0;
}
