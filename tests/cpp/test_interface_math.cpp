// Prints the blade-interface geometry helpers of kynema_b200_interfaces.hpp for
// a few inputs, one value per line, for tests/test_cpp_shim.py to compare with
// independent computations (no GPU: only the header's host code runs).
#include <cstdio>
#include <vector>

#include "kynema_b200_interfaces.hpp"

using namespace kynema_b200::interfaces;

int main() {
    for (size_t order : {1, 4, 10}) {
        for (double x : math::GenerateGLLPoints(order)) std::printf("gll %zu %.17g\n", order, x);
    }
    const std::vector<double> grid{0., 0.1, 0.25, 0.6, 1.};
    for (const auto& q : math::CreateTrapezoidalQuadrature(grid)) std::printf("trap %.17g %.17g\n", q[0], q[1]);
    // a curved axis through 7 key points, fitted by an order-4 element
    std::vector<double> kg;
    std::vector<std::array<double, 3>> kp;
    for (int i = 0; i < 7; ++i) {
        const double s = i / 6.;
        kg.push_back(s);
        kp.push_back({10. * s, 0.5 * s * s, 0.1 * s * s * s});
    }
    const auto nodes = math::FitNodes(math::GenerateGLLPoints(4), kg, kp);
    for (const auto& n : nodes) std::printf("fit %.17g %.17g %.17g\n", n[0], n[1], n[2]);
    const auto q = math::TangentTwistToQuaternion({1., 2., 0.5}, 30.);
    std::printf("ttq %.17g %.17g %.17g %.17g\n", q[0], q[1], q[2], q[3]);
    return 0;
}
