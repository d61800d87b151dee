// The reference's CFD-interface regression tests written against
// kynema_b200_interfaces.hpp: tests/regression_tests/interfaces/test_cfd_interface.cpp
// (PrecessionTest with SaveState / RestoreState, FloatingPlatform with three
// mooring lines, Restart through a restart file), same inputs, same tolerances.
// Exit code 0 on success.
#include <cmath>
#include <cstdio>
#include <numbers>
#include <string>

#include "kynema_b200_interfaces.hpp"

using namespace kynema_b200;
using namespace kynema_b200::interfaces::cfd;

static int failures = 0;
static void expect_near(double a, double b, double tol, const char* what) {
    if (!(std::abs(a - b) <= tol)) {
        std::printf("FAIL %s: %.17g vs %.17g\n", what, a, b);
        ++failures;
    }
}
static void expect_q(const std::array<double, 7>& u, const double (&e)[7], const char* what) {
    for (int c = 0; c < 7; ++c) expect_near(u[c], e[c], 1e-12, what);
}

static void precession(const Context& ctx) {
    const auto mass = std::array{std::array{1., 0., 0., 0., 0., 0.}, std::array{0., 1., 0., 0., 0., 0.},
                                 std::array{0., 0., 1., 0., 0., 0.}, std::array{0., 0., 0., 1., 0., 0.},
                                 std::array{0., 0., 0., 0., 1., 0.}, std::array{0., 0., 0., 0., 0., .5}};
    auto interface = InterfaceBuilder{}
                         .SetTimeStep(0.01)
                         .SetDampingFactor(1.)
                         .SetMaximumNonlinearIterations(5U)
                         .EnableFloatingPlatform(true)
                         .SetFloatingPlatformVelocity({0., 0., 0., 0.5, 0.5, 1.})
                         .SetFloatingPlatformMassMatrix(mass)
                         .Build(ctx);
    const auto& node = interface.turbine.floating_platform.node;
    for (int i = 0; i < 500; ++i)
        if (!interface.Step()) { std::printf("FAIL precession step %d\n", i); ++failures; }
    const double q500[7] = {0., 0., 0., -0.63053045128590757, 0.60556039120583116, -0.30157681970585326,
                            -0.38049886257377241};
    const double q600[7] = {0., 0., 0., -0.35839735533217154, 0.31963488733920042, -0.27587277763126217,
                            -0.83263382410791731};
    expect_q(node.displacement, q500, "precession q at 500");
    interface.SaveState();
    for (int i = 500; i < 600; ++i) interface.Step();
    expect_q(node.displacement, q600, "precession q at 600");
    interface.RestoreState();
    expect_q(node.displacement, q500, "precession q restored to 500");
    for (int i = 500; i < 600; ++i) interface.Step();
    expect_q(node.displacement, q600, "precession q at 600 again");
}

static InterfaceBuilder moored_platform() {
    constexpr double m = 1.419625E+7;
    const auto mass = std::array{std::array{m, 0., 0., 0., 0., 0.}, std::array{0., m, 0., 0., 0., 0.},
                                 std::array{0., 0., m, 0., 0., 0.}, std::array{0., 0., 0., 1.2898E+10, 0., 0.},
                                 std::array{0., 0., 0., 0., 1.2851E+10, 0.}, std::array{0., 0., 0., 0., 0., 1.4189E+10}};
    return InterfaceBuilder{}
        .SetGravity({0., 0., -9.8124})
        .SetTimeStep(0.01)
        .SetDampingFactor(0.)
        .SetMaximumNonlinearIterations(5)
        .EnableFloatingPlatform(true)
        .SetFloatingPlatformPosition({0., 0., -7.53, 1., 0., 0., 0.})
        .SetFloatingPlatformMassMatrix(mass)
        .SetNumberOfMooringLines(3)
        .SetMooringLineStiffness(0, 48.9e3)
        .SetMooringLineUndeformedLength(0, 55.432)
        .SetMooringLineFairleadPosition(0, {-40.87, 0.0, -14.})
        .SetMooringLineAnchorPosition(0, {-105.47, 0.0, -58.4})
        .SetMooringLineStiffness(1, 48.9e3)
        .SetMooringLineUndeformedLength(1, 55.432)
        .SetMooringLineFairleadPosition(1, {20.43, -35.39, -14.})
        .SetMooringLineAnchorPosition(1, {52.73, -91.34, -58.4})
        .SetMooringLineStiffness(2, 48.9e3)
        .SetMooringLineUndeformedLength(2, 55.432)
        .SetMooringLineFairleadPosition(2, {20.43, 35.39, -14.})
        .SetMooringLineAnchorPosition(2, {52.73, 91.34, -58.4});
}

static void floating_platform(const Context& ctx) {
    auto interface = moored_platform().Build(ctx);
    const double spring0 = 1907514.4912628897;
    const double buoyancy = spring0 + 9.8124 * 1.419625E+7;
    auto& node = interface.turbine.floating_platform.node;
    const double w = 2. * std::numbers::pi;
    for (int i = 0; i <= 100; ++i) {
        const double t = 0.01 * i;
        node.loads[1] = 1e6 * std::sin(w / 20. * t);
        node.loads[2] = buoyancy + 0.5 * spring0 * std::sin(w / 20. * t);
        node.loads[3] = 5.0e5 * std::sin(w / 15. * t);
        node.loads[4] = 1.0e6 * std::sin(w / 30. * t);
        node.loads[5] = 2.0e7 * std::sin(w / 60. * t);
        if (!interface.Step()) { std::printf("FAIL floating platform step %d\n", i); ++failures; }
    }
    const double q[7] = {3.4379940641493395e-06, 0.0036709089002912518, 0.0034998271929752248, 0.99999999992274302,
                         1.3448158662549561e-06, 1.2713890988278111e-06, 1.2291853012439073e-05};
    expect_q(node.displacement, q, "floating platform q at step 100");
}

static void restart(const Context& ctx, const std::string& path) {
    const auto builder = moored_platform();
    auto a = builder.Build(ctx);
    auto drive = [](Interface& it) {
        for (int i = 0; i < 100; ++i) {
            it.turbine.floating_platform.node.loads[1] = 1e6 * std::sin(2. * std::numbers::pi / 20. * 0.01 * i);
            if (!it.Step()) { std::printf("FAIL restart step %d\n", i); ++failures; }
        }
    };
    drive(a);
    a.WriteRestart(path);
    drive(a);
    auto b = builder.Build(ctx);
    b.ReadRestart(path);
    drive(b);
    for (int c = 0; c < 7; ++c)
        expect_near(b.turbine.floating_platform.node.displacement[c], a.turbine.floating_platform.node.displacement[c],
                    1e-12, "restart: platform q after 100 more steps");
    std::remove(path.c_str());
}

int main(int argc, char** argv) {
    try {
        Context ctx(0);
        precession(ctx);
        floating_platform(ctx);
        restart(ctx, argc > 1 ? argv[1] : "cfd_interface_restart.dat");
    } catch (const std::exception& e) {
        std::printf("FAIL exception: %s\n", e.what());
        return 2;
    }
    std::printf("%s (%d failures)\n", failures ? "FAILED" : "OK", failures);
    return failures ? 1 : 0;
}
