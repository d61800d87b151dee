// TurbineInterfaceTest.IEA15_Structure
// (tests/regression_tests/interfaces/test_turbine_interface.cpp:17-285) against the
// C++ host shim's turbine interface: the IEA-15-240-RWT structure built from its
// WindIO description (blades from argv[1] = tests/golden/iea15_blade_windio.txt,
// tower, hub and nacelle from argv[2] = tests/golden/iea15_turbine_windio.txt),
// a tower-top load, generator torque, a pitch ramp on blade 3 and a yaw ramp for
// 9 steps of 0.01 s, every step converged, and the tower top position at the
// test's 1e-10.  The oracle (test infrastructure, oracle/kyn_oracle.h) steps the
// same model description beside it: same Newton iteration counts at every step,
// displacements within 1e-10 relative.  Exit code 0 on success.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <numbers>
#include <sstream>
#include <string>
#include <vector>

#include "kyn_oracle.h"
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

static std::istringstream read_fixture(const char* path) {
    std::ifstream in(path);
    if (!in) throw std::runtime_error(std::string("cannot open ") + path);
    std::string line, text;
    while (std::getline(in, line))
        if (line.empty() || line[0] != '#') text += line + "\n";
    return std::istringstream(text);
}

using M6 = std::array<std::array<double, 6>, 6>;

static M6 symmetric(const double* a) {
    return M6{{{a[0], a[1], a[2], a[3], a[4], a[5]},
               {a[1], a[6], a[7], a[8], a[9], a[10]},
               {a[2], a[7], a[11], a[12], a[13], a[14]},
               {a[3], a[8], a[12], a[15], a[16], a[17]},
               {a[4], a[9], a[13], a[16], a[18], a[19]},
               {a[5], a[10], a[14], a[17], a[19], a[20]}}};
}

// the six-by-six point inertia of the test: mass on the translations, the
// WindIO inertia [xx, yy, zz, xy, xz, yz] on the rotations
static M6 point_inertia(double mass, const double* I) {
    return M6{{{mass, 0., 0., 0., 0., 0.},
               {0., mass, 0., 0., 0., 0.},
               {0., 0., mass, 0., 0., 0.},
               {0., 0., 0., I[0], I[3], I[4]},
               {0., 0., 0., I[3], I[1], I[5]},
               {0., 0., 0., I[4], I[5], I[2]}}};
}

int main(int argc, char** argv) {
    if (argc < 3) {
        std::printf("usage: %s <iea15_blade_windio.txt> <iea15_turbine_windio.txt>\n", argv[0]);
        return 2;
    }
    try {
        const double time_step = 0.01, duration = 0.1;
        const size_t n_blades = 3, n_blade_nodes = 11, n_tower_nodes = 11;
        TurbineInterfaceBuilder builder;
        builder.Solution()
            .EnableDynamicSolve()
            .SetTimeStep(time_step)
            .SetDampingFactor(0.0)
            .SetGravity({0., 0., -9.81})
            .SetMaximumNonlinearIterations(6)
            .SetAbsoluteErrorTolerance(1e-6)
            .SetRelativeErrorTolerance(1e-4);
        const auto Z = components::ReferenceAxisOrientation::Z;

        auto tf = read_fixture(argv[2]);
        size_t n = 0;
        std::vector<std::array<double, 4>> tower_axis;
        tf >> n;
        for (size_t i = 0; i < n; ++i) {
            std::array<double, 4> r{};
            tf >> r[0] >> r[1] >> r[2] >> r[3];
            tower_axis.push_back(r);
        }
        std::vector<std::array<double, 3>> tower_stations;
        tf >> n;
        for (size_t i = 0; i < n; ++i) {
            std::array<double, 3> r{};
            tf >> r[0] >> r[1] >> r[2];
            tower_stations.push_back(r);
        }
        double E, G, rho, nu;
        tf >> E >> G >> rho >> nu;
        double hub_diameter, cone_angle, hub_mass, hub_inertia[6];
        tf >> hub_diameter >> cone_angle >> hub_mass;
        for (double& v : hub_inertia) tf >> v;
        double uptilt, overhang, distance_tt_hub, system_mass, yaw_mass, inertia_tt[6];
        tf >> uptilt >> overhang >> distance_tt_hub >> system_mass >> yaw_mass;
        for (double& v : inertia_tt) tf >> v;
        double expected[7];
        for (double& v : expected) tf >> v;
        if (!tf) throw std::runtime_error("truncated turbine fixture");

        auto& turbine_builder = builder.Turbine();
        turbine_builder.SetAzimuthAngle(0.)
            .SetRotorApexToHub(0.)
            .SetHubDiameter(hub_diameter)
            .SetConeAngle(cone_angle)
            .SetShaftTiltAngle(uptilt)
            .SetTowerAxisToRotorApex(overhang)
            .SetTowerTopToRotorApex(distance_tt_hub);

        // blades: the IEA-15 blade of BladeInterfaceTest.BladeWindIO, three times
        for (size_t j = 0; j < n_blades; ++j) {
            auto bf = read_fixture(argv[1]);
            auto& blade = turbine_builder.Blade(j);
            blade.SetElementOrder(n_blade_nodes - 1).PrescribedRootMotion(false);
            bf >> n;
            for (size_t i = 0; i < n; ++i) {
                double g, x, y, z;
                bf >> g >> x >> y >> z;
                blade.AddRefAxisPoint(g, {x, y, z}, Z);
            }
            bf >> n;
            for (size_t i = 0; i < n; ++i) {
                double g, t;
                bf >> g >> t;
                blade.AddRefAxisTwist(g, t * std::numbers::pi / 180.);
            }
            bf >> n;
            for (size_t i = 0; i < n; ++i) {
                double g, m[21], k[21];
                bf >> g;
                for (double& v : m) bf >> v;
                for (double& v : k) bf >> v;
                blade.AddSection(g, symmetric(m), symmetric(k), Z);
            }
            if (!bf) throw std::runtime_error("truncated blade fixture");
        }

        // tower
        auto& tower = turbine_builder.Tower();
        tower.SetElementOrder(n_tower_nodes - 1).PrescribedRootMotion(false);
        for (const auto& r : tower_axis) tower.AddRefAxisPoint(r[0], {r[1], r[2], r[3]}, Z);
        turbine_builder.SetTowerBasePosition(
            {tower_axis[0][1], tower_axis[0][2], tower_axis[0][3], 1., 0., 0., 0.});
        tower.AddRefAxisTwist(0.0, 0.0).AddRefAxisTwist(1.0, 0.0);
        for (const auto& st : tower_stations) {
            const auto section = beams::GenerateHollowCircleSection(st[0], E, G, rho, st[1], st[2], nu);
            tower.AddSection(st[0], section.M_star, section.C_star, Z);
        }

        // nacelle (yaw bearing) and hub masses
        turbine_builder.SetYawBearingInertiaMatrix(point_inertia(system_mass + yaw_mass, inertia_tt));
        turbine_builder.SetHubInertiaMatrix(point_inertia(hub_mass, hub_inertia));

        if (argc > 3 && std::string(argv[3]) == "--describe") {
            // host only (no device): the turbine's model description through
            // kyn_model_describe, its DOF counts and CRS graph against the oracle's
            Model model(builder.Solution().Input().gravity);
            components::Turbine turbine(builder.Turbine().Input(), model);
            model.WithDescription([&](const kyn_model_desc& d) {
                kyn_model_info info{};
                char e[256] = {};
                if (kyn_model_describe(&d, &info, nullptr, nullptr, e, 256) != KYN_OK)
                    throw std::runtime_error(std::string("describe: ") + e);
                std::vector<int32_t> rp(static_cast<size_t>(info.num_dofs) + 1), ci(static_cast<size_t>(info.nnz));
                kyn_model_describe(&d, &info, rp.data(), ci.data(), e, 256);
                orc_model* o = orc_model_create(&d, e, 256);
                if (!o) throw std::runtime_error(std::string("oracle: ") + e);
                kyn_model_info oi{};
                orc_model_info(o, &oi);
                std::vector<int> orp(static_cast<size_t>(oi.num_dofs) + 1), oci(static_cast<size_t>(oi.nnz));
                orc_get_crs(o, orp.data(), oci.data(), nullptr);
                orc_model_destroy(o);
                std::printf("describe: %d nodes, %d constraints, %d unknowns, %d in the condensed system, nnz %d\n",
                            info.num_nodes, info.num_constraints, info.num_dofs, info.condensed_dofs, info.nnz);
                bool same = info.num_dofs == oi.num_dofs && info.nnz == oi.nnz;
                for (size_t k = 0; same && k < rp.size(); ++k) same = rp[k] == orp[k];
                for (size_t k = 0; same && k < ci.size(); ++k) same = ci[k] == oci[k];
                if (!same || info.num_dofs != 371 || info.condensed_dofs != 137) {
                    std::printf("FAIL the turbine's DOF counts or CRS graph differ from the oracle's\n");
                    ++failures;
                }
            });
            std::printf("%s\n", failures ? "FAILED" : "OK");
            return failures ? 1 : 0;
        }

        auto interface = builder.Build(Context(0));

        // the oracle on the same model description
        orc_model* orc = nullptr;
        char err[256] = {};
        interface.GetModel().WithDescription([&](const kyn_model_desc& d) { orc = orc_model_create(&d, err, 256); });
        if (!orc) throw std::runtime_error(std::string("oracle: ") + err);
        kyn_model_info oinfo{};
        orc_model_info(orc, &oinfo);
        std::vector<double> f(static_cast<size_t>(oinfo.num_nodes) * 6, 0.);
        const StepParameters sp(true, 6, time_step, 0.0, 1e-6, 1e-4);
        const kyn_step_params op = sp.c();

        auto& t = interface.Turbine();
        t.tower.nodes.back().loads = {1e5, 0., 0., 0., 0., 0.};
        t.torque_control = 1e8;
        const auto n_steps = static_cast<size_t>(duration / time_step);
        double worst = 0., gpu_s = 0., orc_s = 0., first_s = 0.;
        for (size_t i = 1; i < n_steps; ++i) {
            const double time = static_cast<double>(i) * time_step;
            t.blade_pitch_control[2] = time * 0.5;
            t.yaw_control = time * 0.3;
            if (i % 500 == 0) t.torque_control = 0.;
            const auto g0 = std::chrono::steady_clock::now();
            const bool converged = interface.Step();
            const double dt = std::chrono::duration<double>(std::chrono::steady_clock::now() - g0).count();
            if (i == 1) first_s = dt;
            else gpu_s += dt;
            if (!converged) {
                std::printf("FAIL step %zu did not converge\n", i);
                ++failures;
                break;
            }
            // oracle: the same loads and control inputs, one step
            std::fill(f.begin(), f.end(), 0.);
            for (int c = 0; c < 6; ++c) f[t.tower.nodes.back().id * 6 + c] = t.tower.nodes.back().loads[c];
            orc_set_loads(orc, KYN_LOAD_STATE_F, f.data());
            auto control = [&](size_t cid, double value) {
                const double u[7] = {value, 0., 0., 1., 0., 0., 0.};
                orc_set_prescribed(orc, static_cast<int>(cid), u);
            };
            for (size_t j = 0; j < n_blades; ++j) control(t.blade_pitch[j].id, t.blade_pitch_control[j]);
            control(t.tower_top_to_yaw_bearing.id, t.yaw_control);
            control(t.shaft_base_to_azimuth.id, t.torque_control);
            int oit = 0;
            const auto o0 = std::chrono::steady_clock::now();
            const int ost = orc_step(orc, &op, &oit);
            orc_s += std::chrono::duration<double>(std::chrono::steady_clock::now() - o0).count();
            const int git = static_cast<int>(interface.GetSolver().convergence_err().size());
            if (ost != KYN_OK || oit != git) {
                std::printf("FAIL step %zu: oracle status %d iterations %d, GPU iterations %d\n", i, ost, oit, git);
                ++failures;
            }
            std::vector<double> oq(static_cast<size_t>(oinfo.num_nodes) * 7);
            orc_get_state(orc, KYN_FIELD_Q, oq.data());
            std::vector<double> gq(oq.size());
            const auto gx = interface.GetSolver().model();
            check(gx->ctx.get(), kyn_get_state(gx->ctx.get(), gx->id, KYN_FIELD_Q, gq.data()));
            double scale = 0., diff = 0.;
            for (size_t k = 0; k < oq.size(); ++k) {
                scale = std::max(scale, std::abs(oq[k]));
                diff = std::max(diff, std::abs(oq[k] - gq[k]));
            }
            worst = std::max(worst, diff / scale);
        }
        std::printf("oracle: largest relative difference of q over the steps %.3g\n", worst);
        // wall time per step: TurbineInterface::Step (loads and controls in, one
        // condensed dense step on the GPU, motion out; the first step, which
        // also loads the kernel and builds the launch plan, apart) and the
        // oracle's step (one core)
        std::printf("time per step: interface %.3f ms (first step %.3f ms), oracle %.3f ms\n",
                    1e3 * gpu_s / (n_steps - 2), 1e3 * first_s, 1e3 * orc_s / (n_steps - 1));
        if (!(worst <= 1e-10)) {
            std::printf("FAIL q differs from the oracle by %.3g relative\n", worst);
            ++failures;
        }
        {  // the shaft joint's output: azimuth angle and rotor speed
            std::vector<double> oo(static_cast<size_t>(oinfo.num_constraints) * 3);
            orc_get_state(orc, KYN_FIELD_CONSTRAINT_OUTPUT, oo.data());
            const size_t rj = t.shaft_base_to_azimuth.id;
            double az = std::fmod(oo[rj * 3], 2. * std::numbers::pi);
            if (az < 0.) az += 2. * std::numbers::pi;
            expect_near(interface.CalculateAzimuthAngle(), az, 1e-10, "azimuth angle", 0);
            expect_near(interface.CalculateRotorSpeed(), oo[rj * 3 + 1], 1e-10 * (1. + std::abs(oo[rj * 3 + 1])),
                        "rotor speed", 0);
            if (!(std::abs(interface.CalculateRotorSpeed()) > 1e-3)) {
                std::printf("FAIL the generator torque did not turn the rotor\n");
                ++failures;
            }
            std::printf("azimuth %.6g rad, rotor speed %.6g rad/s\n", interface.CalculateAzimuthAngle(),
                        interface.CalculateRotorSpeed());
        }
        orc_model_destroy(orc);

        // throughput: 148 copies of the turbine (one per SM of a B200) stepped by
        // one batched call, from the state the test left
        {
            const auto dm = interface.GetSolver().model();
            kyn_ctx* c = dm->ctx.get();
            std::vector<int> ids;
            for (int k = 0; k < 148; ++k) {
                const int cid = kyn_model_clone(c, dm->id);
                check(c, cid);
                ids.push_back(cid);
            }
            const kyn_step_params bp = sp.c();
            std::vector<int> st(ids.size()), it(ids.size());
            check(c, kyn_step(c, ids.data(), static_cast<int>(ids.size()), &bp, st.data(), it.data()));
            const int reps = 5;
            const auto b0 = std::chrono::steady_clock::now();
            for (int r = 0; r < reps; ++r)
                check(c, kyn_step(c, ids.data(), static_cast<int>(ids.size()), &bp, st.data(), it.data()));
            const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - b0).count();
            int converged = 0;
            for (int s2 : st) converged += s2 == KYN_OK;
            std::printf("batch of %zu turbines: %.3f ms per batched step, %.0f turbine-steps/s (%d converged)\n",
                        ids.size(), 1e3 * sec / reps, ids.size() * reps / sec, converged);
            // per-phase SM cycles of one more batched step (KYN_OPT_PHASE_TIMING),
            // per turbine and Newton iteration
            check(c, kyn_ctx_set_option(c, KYN_OPT_PHASE_TIMING, 1));
            check(c, kyn_step(c, ids.data(), static_cast<int>(ids.size()), &bp, st.data(), it.data()));
            long iters = 0;
            for (int v : it) iters += v;
            const char* names[] = {"predict+tangent", "(elements: quadrature)", "elements", "bordered assembly", "",
                                   "bordered LU", "back substitution", "update", "", "(elements: assembly)",
                                   "(elements: elimination)", "(elements: save)"};
            std::printf("phase cycles per turbine-iteration (%ld iterations):", iters);
            for (int ph : {0, 2, 1, 9, 10, 11, 3, 5, 6, 7}) {
                int64_t v = 0;
                check(c, kyn_ctx_stat(c, KYN_STAT_PHASE_CYCLES + ph, &v));
                std::printf(" %s %.0f,", names[ph], static_cast<double>(v) / static_cast<double>(iters));
            }
            std::printf("\n");
            check(c, kyn_ctx_set_option(c, KYN_OPT_PHASE_TIMING, 0));
            for (int cid : ids) kyn_model_destroy(c, cid);
        }

        const auto& top = t.tower.nodes.back();
        for (int c = 0; c < 7; ++c) expect_near(top.position[c], expected[c], 1e-10, "tower top position", c);
    } catch (const std::exception& e) {
        std::printf("FAIL exception: %s\n", e.what());
        return 1;
    }
    std::printf("%s\n", failures ? "FAILED" : "OK");
    return failures ? 1 : 0;
}
