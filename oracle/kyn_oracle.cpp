// kyn_oracle.cpp -- CPU FP64 oracle for the per-step beam path.
//
// TEST INFRASTRUCTURE ONLY: the checker for the CUDA path and the timed CPU
// baseline.  It restates the reference (Kynema) algorithm in the reference's
// own operation order so that results can be compared at the 1e-13 level of
// the reference's regression tests.  Each function cites the reference file it
// follows; paths are relative to the reference project root.
//
// Third-party arithmetic restated here (not vendored by the reference,
// versions not pinned): KokkosKernels SerialGemm / SerialGemv / serial_axpy /
// serial_nrm2 (textbook loops: C = beta*C; C(i,j) += alpha * sum_p A(i,p)B(p,j)),
// KokkosSparse::sort_crs_graph (per-row ascending sort) and findRelOffset
// (position of a column in a sorted row).  The sparse direct solve (KLU /
// SuperLU / cuDSS) is replaced by a dense LU with partial pivoting; its result
// is pinned end to end by test_solver.cpp and test_rotor.cpp.

#include "kyn_oracle.h"

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <numeric>
#include <string>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// Floating-point operation tally of the quadrature-point physics (a6-a10),
// compiled in only with -DORC_COUNT_FLOPS (oracle/_build/libkyn_oracle_flops.so):
// every add, subtract, multiply, divide and square root of the functions below
// in their operation order, so that the per-point count the roofline uses is
// counted from this restatement of the reference rather than estimated.
#ifdef ORC_COUNT_FLOPS
long long g_flops = 0;     // every counted operation
long long g_qp_flops = 0;  // those of the quadrature-point loops of update_beam
#define ORC_FLOPS(n) (g_flops += static_cast<long long>(n))
#else
#define ORC_FLOPS(n) ((void)0)
#endif

using V3 = std::array<double, 3>;
using V4 = std::array<double, 4>;
using M3 = std::array<double, 9>;
using M6 = std::array<double, 36>;

// KokkosBatched::SerialGemm restated (row-major, strided, optional transposes).
void gemm(bool ta, bool tb, int m, int n, int k, double alpha, const double* A, int lda,
          const double* B, int ldb, double beta, double* C, int ldc) {
    ORC_FLOPS((beta != 0. && beta != 1. ? m * n : 0) + (alpha != 0. ? 2 * m * n * k + 2 * m * n : 0));
    if (beta == 0.) {
        for (int i = 0; i < m; ++i)
            for (int j = 0; j < n; ++j) C[i * ldc + j] = 0.;
    } else if (beta != 1.) {
        for (int i = 0; i < m; ++i)
            for (int j = 0; j < n; ++j) C[i * ldc + j] *= beta;
    }
    if (alpha == 0.) return;
    for (int i = 0; i < m; ++i) {
        for (int j = 0; j < n; ++j) {
            double c = 0.;
            for (int p = 0; p < k; ++p) {
                const double a = ta ? A[p * lda + i] : A[i * lda + p];
                const double b = tb ? B[j * ldb + p] : B[p * ldb + j];
                c += a * b;
            }
            C[i * ldc + j] += alpha * c;
        }
    }
}

// KokkosBlas::SerialGemv restated: y = beta*y; y(i) += alpha * sum_j op(A)(i,j) x(j).
void gemv(bool ta, int m, int n, double alpha, const double* A, int lda, const double* x,
          double beta, double* y) {
    ORC_FLOPS((beta != 0. && beta != 1. ? m : 0) + (alpha != 0. ? 2 * m * n + 2 * m : 0));
    if (beta == 0.) {
        for (int i = 0; i < m; ++i) y[i] = 0.;
    } else if (beta != 1.) {
        for (int i = 0; i < m; ++i) y[i] *= beta;
    }
    if (alpha == 0.) return;
    for (int i = 0; i < m; ++i) {
        double t = 0.;
        for (int j = 0; j < n; ++j) t += (ta ? A[j * lda + i] : A[i * lda + j]) * x[j];
        y[i] += alpha * t;
    }
}

// src/math/vector_operations.hpp:11-21 VecTilde
M3 tilde(const double* v) {
    return M3{0., -v[2], v[1], v[2], 0., -v[0], -v[1], v[0], 0.};
}

// src/math/quaternion_operations.hpp:20-32 QuaternionToRotationMatrix
M3 quat_to_rot(const double* q) {
    ORC_FLOPS(45);  // 3 diagonal entries x 7, 6 off-diagonal x 4
    return M3{q[0] * q[0] + q[1] * q[1] - q[2] * q[2] - q[3] * q[3],
              2. * (q[1] * q[2] - q[0] * q[3]),
              2. * (q[1] * q[3] + q[0] * q[2]),
              2. * (q[1] * q[2] + q[0] * q[3]),
              q[0] * q[0] - q[1] * q[1] + q[2] * q[2] - q[3] * q[3],
              2. * (q[2] * q[3] - q[0] * q[1]),
              2. * (q[1] * q[3] - q[0] * q[2]),
              2. * (q[2] * q[3] + q[0] * q[1]),
              q[0] * q[0] - q[1] * q[1] - q[2] * q[2] + q[3] * q[3]};
}

// src/math/quaternion_operations.hpp:118-129 RotateVectorByQuaternion
V3 rotate_vec(const double* q, const double* v) {
    ORC_FLOPS(60);  // per component: 8 (diagonal term) + 2 x 5 (off-diagonal) + 2 adds
    V3 r;
    r[0] = (q[0] * q[0] + q[1] * q[1] - q[2] * q[2] - q[3] * q[3]) * v[0] +
           2. * (q[1] * q[2] - q[0] * q[3]) * v[1] + 2. * (q[1] * q[3] + q[0] * q[2]) * v[2];
    r[1] = 2. * (q[1] * q[2] + q[0] * q[3]) * v[0] +
           (q[0] * q[0] - q[1] * q[1] + q[2] * q[2] - q[3] * q[3]) * v[1] +
           2. * (q[2] * q[3] - q[0] * q[1]) * v[2];
    r[2] = 2. * (q[1] * q[3] - q[0] * q[2]) * v[0] + 2. * (q[2] * q[3] + q[0] * q[1]) * v[1] +
           (q[0] * q[0] - q[1] * q[1] - q[2] * q[2] + q[3] * q[3]) * v[2];
    return r;
}

// src/math/quaternion_operations.hpp:204-211 QuaternionCompose
V4 quat_compose(const double* a, const double* b) {
    ORC_FLOPS(28);  // 16 multiplies, 12 adds
    return V4{a[0] * b[0] - a[1] * b[1] - a[2] * b[2] - a[3] * b[3],
              a[0] * b[1] + a[1] * b[0] + a[2] * b[3] - a[3] * b[2],
              a[0] * b[2] - a[1] * b[3] + a[2] * b[0] + a[3] * b[1],
              a[0] * b[3] + a[1] * b[2] - a[2] * b[1] + a[3] * b[0]};
}

// src/math/quaternion_operations.hpp:176-186 QuaternionInverse (device form)
V4 quat_inverse(const double* q) {
    const double len = std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
    return V4{q[0] / len, -q[1] / len, -q[2] / len, -q[3] / len};
}

// src/math/quaternion_operations.hpp:231-242 RotationVectorToQuaternion (device form)
V4 rotvec_to_quat(const double* phi) {
    const double angle = std::sqrt(phi[0] * phi[0] + phi[1] * phi[1] + phi[2] * phi[2]);
    const double cos_angle = std::cos(angle / 2.);
    const double factor = (std::abs(angle) < 1.e-12) ? 0. : std::sin(angle / 2.) / angle;
    return V4{cos_angle, phi[0] * factor, phi[1] * factor, phi[2] * factor};
}

// src/math/quaternion_operations.hpp:153-166 QuaternionDerivative (3x4)
std::array<double, 12> quat_derivative(const double* q) {
    return {-q[1], q[0], -q[3], q[2], -q[2], q[3], q[0], -q[1], -q[3], -q[2], q[1], q[0]};
}

// src/math/matrix_operations.hpp:19-33 AX_Matrix
M3 ax_matrix(const M3& A) {
    double trace = 0.;
    for (int i = 0; i < 3; ++i) trace += A[i * 4];
    trace /= 2.;
    M3 out{};
    for (int i = 0; i < 3; ++i) {
        for (int j = 0; j < 3; ++j) out[i * 3 + j] = -A[i * 3 + j] / 2.;
        out[i * 4] += trace;
    }
    return out;
}

// src/math/matrix_operations.hpp:47-51 AxialVectorOfMatrix
V3 axial(const M3& m) {
    return V3{(m[7] - m[5]) / 2., (m[2] - m[6]) / 2., (m[3] - m[1]) / 2.};
}

double nrm2(const double* v, int n) {
    ORC_FLOPS(2 * n + 1);
    double s = 0.;
    for (int i = 0; i < n; ++i) s += v[i] * v[i];
    return std::sqrt(s);
}

// src/system/masses/rotate_section_matrix.hpp:17-51 RotateSectionMatrix
void rotate_section(const double* xr, const double* cstar, double* cuu) {
    const M3 R = quat_to_rot(xr);
    M6 tmp{};
    gemm(false, false, 3, 6, 3, 1., R.data(), 3, cstar, 6, 0., tmp.data(), 6);
    gemm(false, false, 3, 6, 3, 1., R.data(), 3, cstar + 18, 6, 0., tmp.data() + 18, 6);
    gemm(false, true, 6, 3, 3, 1., tmp.data(), 6, R.data(), 3, 0., cuu, 6);
    gemm(false, true, 6, 3, 3, 1., tmp.data() + 3, 6, R.data(), 3, 0., cuu + 3, 6);
}

// src/system/masses/calculate_inertial_force.hpp:16-53 CalculateInertialForce
void inertial_force(double mass, const double* uddot, const double* omega, const double* omegadot,
                    const double* eta, const M3& eta_t, const M3& rho, const M3& om_t,
                    const M3& omd_t, double* FI) {
    M3 M1{};
    V3 V1{};
    gemm(false, false, 3, 3, 3, mass, om_t.data(), 3, om_t.data(), 3, 0., M1.data(), 3);
    ORC_FLOPS(18 + 6 + 6);  // the three axpy loops of this function
    for (int i = 0; i < 9; ++i) M1[i] += mass * omd_t[i];
    gemv(false, 3, 3, 1., M1.data(), 3, eta, 0., FI);
    for (int i = 0; i < 3; ++i) FI[i] += mass * uddot[i];
    for (int i = 0; i < 3; ++i) V1[i] += mass * uddot[i];
    gemv(false, 3, 3, 1., eta_t.data(), 3, V1.data(), 0., FI + 3);
    gemv(false, 3, 3, 1., rho.data(), 3, omegadot, 1., FI + 3);
    gemm(false, false, 3, 3, 3, 1., om_t.data(), 3, rho.data(), 3, 0., M1.data(), 3);
    gemv(false, 3, 3, 1., M1.data(), 3, omega, 1., FI + 3);
}

// src/system/masses/calculate_gravity_force.hpp:15-27 CalculateGravityForce
void gravity_force(double mass, const double* g, const M3& eta_t, double* FG) {
    ORC_FLOPS(6);
    for (int i = 0; i < 6; ++i) FG[i] = 0.;
    for (int i = 0; i < 3; ++i) FG[i] += mass * g[i];
    gemv(false, 3, 3, 1., eta_t.data(), 3, FG, 0., FG + 3);
}

// src/system/masses/calculate_gyroscopic_matrix.hpp:20-60 CalculateGyroscopicMatrix
void gyroscopic_matrix(double mass, const double* omega, const double* eta, const M3& rho,
                       const M3& om_t, double* Guu) {
    V3 V1{}, V2{};
    ORC_FLOPS(6);
    for (int i = 0; i < 36; ++i) Guu[i] = 0.;
    for (int i = 0; i < 3; ++i) V1[i] += mass * eta[i];
    gemv(false, 3, 3, 1., om_t.data(), 3, V1.data(), 0., V2.data());
    M3 M1 = tilde(V2.data());
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) Guu[i * 6 + 3 + j] = M1[j * 3 + i];
    M1 = tilde(V1.data());
    gemm(false, true, 3, 3, 3, 1., om_t.data(), 3, M1.data(), 3, 1., Guu + 3, 6);
    gemv(false, 3, 3, 1., rho.data(), 3, omega, 0., V1.data());
    M1 = tilde(V1.data());
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) Guu[(3 + i) * 6 + 3 + j] = M1[i * 3 + j];
    gemm(false, false, 3, 3, 3, 1., om_t.data(), 3, rho.data(), 3, -1., Guu + 21, 6);
}

// src/system/masses/calculate_inertia_stiffness_matrix.hpp:19-60
void inertia_stiffness_matrix(double mass, const double* uddot, const double* omegadot,
                              const double* omega, const double* eta, const M3& rho,
                              const M3& om_t, const M3& omd_t, double* Kuu) {
    V3 V1{};
    M3 M1{}, M2{};
    ORC_FLOPS(18 + 6 + 18);  // the three axpy loops of this function
    for (int i = 0; i < 36; ++i) Kuu[i] = 0.;
    for (int i = 0; i < 9; ++i) M1[i] += 1. * omd_t[i];
    gemm(false, false, 3, 3, 3, 1., om_t.data(), 3, om_t.data(), 3, 1., M1.data(), 3);
    for (int i = 0; i < 3; ++i) V1[i] += mass * eta[i];
    M2 = tilde(V1.data());
    gemm(false, true, 3, 3, 3, 1., M1.data(), 3, M2.data(), 3, 0., Kuu + 3, 6);
    M1 = tilde(uddot);
    gemm(false, false, 3, 3, 3, 1., rho.data(), 3, omd_t.data(), 3, 0., Kuu + 21, 6);
    gemm(false, false, 3, 3, 3, 1., M1.data(), 3, M2.data(), 3, 1., Kuu + 21, 6);
    gemv(false, 3, 3, 1., rho.data(), 3, omegadot, 0., V1.data());
    M2 = tilde(V1.data());
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) Kuu[(3 + i) * 6 + 3 + j] += -1. * M2[i * 3 + j];
    gemv(false, 3, 3, 1., rho.data(), 3, omega, 0., V1.data());
    M1 = tilde(V1.data());
    gemm(false, false, 3, 3, 3, 1., rho.data(), 3, om_t.data(), 3, -1., M1.data(), 3);
    gemm(false, false, 3, 3, 3, 1., om_t.data(), 3, M1.data(), 3, 1., Kuu + 21, 6);
}

// src/system/beams/calculate_inertial_quadrature_point_values.hpp:44-126
// (from the QuaternionCompose(r, r0) onward; r already interpolated and normalised)
void inertial_qp(const double* mstar, const double* r0, const double* r, const double* uddot,
                 const double* omega, const double* omegadot, const double* g, double* FI,
                 double* FG, double* Muu, double* Guu, double* Kuu) {
    const V4 xr = quat_compose(r, r0);
    rotate_section(xr.data(), mstar, Muu);
    const double mass = Muu[0];
    ORC_FLOPS(3);  // eta
    // src/system/masses/calculate_mass_matrix_components.hpp CalculateEta / CalculateRho
    const V3 eta{Muu[5 * 6 + 1] / mass, -Muu[5 * 6 + 0] / mass, Muu[4 * 6 + 0] / mass};
    const M3 eta_t = tilde(eta.data());
    M3 rho;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) rho[i * 3 + j] = Muu[(3 + i) * 6 + 3 + j];
    const M3 om_t = tilde(omega);
    const M3 omd_t = tilde(omegadot);
    inertial_force(mass, uddot, omega, omegadot, eta.data(), eta_t, rho, om_t, omd_t, FI);
    gravity_force(mass, g, eta_t, FG);
    gyroscopic_matrix(mass, omega, eta.data(), rho, om_t, Guu);
    inertia_stiffness_matrix(mass, uddot, omegadot, omega, eta.data(), rho, om_t, omd_t, Kuu);
}

// src/system/beams/calculate_strain.hpp:17-47
void calc_strain(const double* x0p, const double* up, const double* r, const double* rp,
                 double* strain) {
    V3 R = rotate_vec(r, x0p);
    ORC_FLOPS(12);
    for (int i = 0; i < 3; ++i) R[i] += -1. * up[i];
    for (int i = 0; i < 3; ++i) R[i] += -1. * x0p[i];
    const auto E = quat_derivative(r);
    double e2[3];
    gemv(false, 3, 4, 2., E.data(), 4, rp, 0., e2);
    strain[0] = -R[0];
    strain[1] = -R[1];
    strain[2] = -R[2];
    strain[3] = e2[0];
    strain[4] = e2[1];
    strain[5] = e2[2];
}

// src/system/beams/calculate_Ouu.hpp:17-37
void calc_ouu(const double* cuu, const double* ss, const double* mt, const double* nt,
              double* O) {
    ORC_FLOPS(36);
    for (int i = 0; i < 36; ++i) O[i] = 0.;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) O[i * 6 + 3 + j] += 1. * nt[i * 3 + j];
    gemm(false, false, 3, 3, 3, 1., cuu, 6, ss, 3, -1., O + 3, 6);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) O[(3 + i) * 6 + 3 + j] += 1. * mt[i * 3 + j];
    gemm(false, false, 3, 3, 3, 1., cuu + 18, 6, ss, 3, -1., O + 21, 6);
}

// src/system/beams/calculate_Puu.hpp:17-36
void calc_puu(const double* cuu, const double* ss, const double* nt, double* P) {
    ORC_FLOPS(18);
    for (int i = 0; i < 36; ++i) P[i] = 0.;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) P[(3 + i) * 6 + j] += 1. * nt[i * 3 + j];
    gemm(true, false, 3, 3, 3, 1., ss, 3, cuu, 6, 1., P + 18, 6);
    gemm(true, false, 3, 3, 3, 1., ss, 3, cuu + 3, 6, 0., P + 21, 6);
}

// src/system/beams/calculate_Quu.hpp:17-38
void calc_quu(const double* cuu, const double* ss, const double* nt, double* Qm) {
    M3 M1{};
    ORC_FLOPS(18);
    for (int i = 0; i < 36; ++i) Qm[i] = 0.;
    for (int i = 0; i < 9; ++i) M1[i] += 1. * nt[i];
    gemm(false, false, 3, 3, 3, 1., cuu, 6, ss, 3, -1., M1.data(), 3);
    gemm(true, false, 3, 3, 3, 1., ss, 3, M1.data(), 3, 0., Qm + 21, 6);
}

// src/system/beams/calculate_stiffness_quadrature_point_values.hpp:47-128
void stiffness_qp(const double* cstar, const double* r0, const double* x0p, const double* up,
                  const double* r, const double* rp, double* FC, double* FD, double* Cuu,
                  double* Ouu, double* Puu, double* Quu) {
    const V4 xr = quat_compose(r, r0);
    rotate_section(xr.data(), cstar, Cuu);
    double strain[6];
    calc_strain(x0p, up, r, rp, strain);
    // calculate_temporary_variables.hpp:17-28
    double x0pup[3] = {x0p[0], x0p[1], x0p[2]};
    ORC_FLOPS(6);
    for (int i = 0; i < 3; ++i) x0pup[i] += 1. * up[i];
    const M3 ss = tilde(x0pup);
    // calculate_force_FC.hpp / calculate_force_FD.hpp
    gemv(false, 6, 6, 1., Cuu, 6, strain, 0., FC);
    for (int i = 0; i < 6; ++i) FD[i] = 0.;
    gemv(true, 3, 3, 1., ss.data(), 3, FC, 0., FD + 3);
    const M3 nt = tilde(FC);
    const M3 mt = tilde(FC + 3);
    calc_ouu(Cuu, ss.data(), mt.data(), nt.data(), Ouu);
    calc_puu(Cuu, ss.data(), nt.data(), Puu);
    calc_quu(Cuu, ss.data(), nt.data(), Quu);
}

// src/system/calculate_tangent_operator.hpp:26-65 (output stored transposed)
void tangent_operator(double h, const double* qd, double* Tg) {
    M6 T{};
    for (int k = 0; k < 6; ++k) T[k * 7] = 1.;
    double rv[3] = {0., 0., 0.};
    for (int i = 0; i < 3; ++i) rv[i] += h * qd[3 + i];
    const double phi = nrm2(rv, 3);
    const double tmp1 = (phi > 1.e-16) ? (std::cos(phi) - 1.) / (phi * phi) : 0.;
    const double tmp2 = (phi > 1.e-16) ? (1. - std::sin(phi) / phi) / (phi * phi) : 0.;
    const M3 m2 = tilde(rv);
    M3 m1 = m2;
    gemm(false, false, 3, 3, 3, tmp2, m2.data(), 3, m2.data(), 3, tmp1, m1.data(), 3);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) T[(3 + i) * 6 + 3 + j] += 1. * m1[i * 3 + j];
    for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j) Tg[i * 6 + j] = T[j * 6 + i];
}

// src/math/interpolation.hpp LagrangePolynomialInterpWeights
void lagrange_interp(double x, const std::vector<double>& xs, std::vector<double>& w) {
    const size_t n = xs.size();
    w.assign(n, 1.);
    std::vector<double> xm(n);
    for (size_t m = 0; m < n; ++m) xm[m] = x - xs[m];
    for (size_t j = 0; j < n; ++j)
        for (size_t m = 0; m < n; ++m)
            if (j != m) w[j] *= xm[m] / (xs[j] - xs[m]);
}

// src/math/interpolation.hpp LagrangePolynomialDerivWeights
void lagrange_deriv(double x, const std::vector<double>& xs, std::vector<double>& w) {
    const size_t n = xs.size();
    w.assign(n, 0.);
    for (size_t i = 0; i < n; ++i) {
        const double xi = xs[i];
        double weight = 0.;
        for (size_t j = 0; j < n; ++j) {
            if (j == i) continue;
            double prod = 1.;
            for (size_t k = 0; k < n; ++k) {
                if (k == i || k == j) continue;
                prod = prod * ((x - xs[k]) / (xi - xs[k]));
            }
            weight += prod / (xi - xs[j]);
        }
        w[i] = weight;
    }
}

// src/math/interpolation.hpp LinearInterpWeights
void linear_interp(double x, const std::vector<double>& xs, std::vector<double>& w) {
    const size_t n = xs.size();
    w.assign(n, 0.);
    const auto lower = std::lower_bound(xs.begin(), xs.end(), x);
    if (lower == xs.begin()) {
        w.front() = 1.;
        return;
    }
    if (lower == xs.end()) {
        w.back() = 1.;
        return;
    }
    const auto index = static_cast<size_t>(std::distance(xs.begin(), lower));
    const double lo = xs[index - 1];
    const double hi = xs[index];
    const double wu = (x - lo) / (hi - lo);
    w[index - 1] = 1. - wu;
    w[index] = wu;
}

int count_bits(unsigned sig) {
    int c = 0;
    for (unsigned v = sig; v > 0; v >>= 1) c += static_cast<int>(v & 1U);
    return c;
}

}  // namespace

// ---------------------------------------------------------------------------
// Model
// ---------------------------------------------------------------------------

struct OBeam {
    int N = 0, Q = 0;
    std::vector<int> node_ids;
    std::vector<double> phi, dphi;      // [N][Q]
    std::vector<double> w, jac;         // [Q]
    std::vector<double> x0p;            // [Q][3]
    std::vector<double> r0;             // [Q][4]
    std::vector<double> mstar, cstar;   // [Q][36]
    std::vector<double> fx;             // [N][6]  node_FX
    std::vector<double> fe;             // [Q][6]  qp_Fe (zero)
    std::vector<double> residual;       // [N][6]
    std::vector<double> sysmat;         // [N][N][36]
    std::vector<long> eft;              // [N][6]
};

// src/elements/masses/masses.hpp: one 6x6 mass at a node
struct OMass {
    int node = 0;
    double mstar[36] = {};
    double r0[4] = {1., 0., 0., 0.};   // node x0 rotation
    double residual[6] = {};
    double sysmat[36] = {};
    long eft[6] = {};
};

// src/elements/springs/springs.hpp: translational spring between two nodes
struct OSpring {
    int n1 = 0, n2 = 0;
    double x0[3] = {};                 // x0(node 2) - x0(node 1)
    double l_ref = 0., k = 0.;
    double residual[2][3] = {};
    double stiff[2][2][9] = {};
    long eft[2][3] = {};
};

struct OConstraint {
    int type = 0;
    int base = 0, target = 0;
    double X0[3] = {0., 0., 0.};
    double axis[3] = {0., 0., 0.};   // RotationControl: axes row 0 (unit axis)
    double axes[9] = {};             // RevoluteJoint: joint frame, row 0 = joint axis
    double output[3] = {0., 0., 0.}; // RevoluteJoint: rotation, rate, acceleration
    double input[7] = {0., 0., 0., 1., 0., 0., 0.};
    double lambda[6] = {0., 0., 0., 0., 0., 0.};
    double res[6] = {};
    double t_lambda_res[6] = {};
    double sys_res[6] = {};
    double t_grad_tan[36] = {};
    double t_grad_trans[36] = {};
    double b_grad_tan[36] = {};      // rigid joint: base-node blocks
    double b_grad_trans[36] = {};
    double b_lambda_res[6] = {};
    long row_first = 0, row_last = 0;
    long base_active = 0, target_active = 0;
    long base_table[6] = {};
    long target_table[6] = {};
};

struct orc_model {
    int num_nodes = 0;
    std::vector<double> x0, x, q, q_prev, q_delta, v, vd, a, f, tangent;
    std::vector<unsigned> sig;
    std::vector<long> active, fmap;
    std::vector<OBeam> beams;
    std::vector<OMass> masses;
    std::vector<OSpring> springs;
    std::vector<OConstraint> cons;
    double gravity[3] = {0., 0., 0.};
    long nsys = 0, ndofs = 0;
    std::vector<long> row_ptrs, col_inds;
    std::vector<double> values, b, xsol;
    std::vector<double> conv;
    int solver_mode = 0;
};

namespace {

// src/state/calculate_next_state.hpp:27-37
void calculate_next_state(orc_model& m, double h, double af, double am, double beta,
                          double gamma) {
    for (int n = 0; n < m.num_nodes; ++n) {
        for (int c = 0; c < 6; ++c) {
            const double v_p = m.v[n * 6 + c];
            const double vd_p = m.vd[n * 6 + c];
            const double a_p = m.a[n * 6 + c];
            m.vd[n * 6 + c] = 0.;
            m.a[n * 6 + c] = (af * vd_p - am * a_p) / (1. - am);
            m.v[n * 6 + c] = v_p + h * (1. - gamma) * a_p + gamma * h * m.a[n * 6 + c];
            m.q_delta[n * 6 + c] = v_p + (0.5 - beta) * h * a_p + beta * h * m.a[n * 6 + c];
        }
    }
}

// src/state/calculate_displacement.hpp:25-50
void calculate_displacement(orc_model& m, double h) {
    for (int n = 0; n < m.num_nodes; ++n) {
        for (int c = 0; c < 3; ++c)
            m.q[n * 7 + c] = m.q_prev[n * 7 + c] + h * m.q_delta[n * 6 + c];
        const double delta[3] = {h * m.q_delta[n * 6 + 3], h * m.q_delta[n * 6 + 4],
                                 h * m.q_delta[n * 6 + 5]};
        const V4 qd = rotvec_to_quat(delta);
        const V4 qn = quat_compose(qd.data(), &m.q_prev[n * 7 + 3]);
        for (int c = 0; c < 4; ++c) m.q[n * 7 + 3 + c] = qn[c];
    }
}

// src/state/update_global_position.hpp:25-45
void update_global_position(orc_model& m) {
    for (int n = 0; n < m.num_nodes; ++n) {
        for (int c = 0; c < 3; ++c) m.x[n * 7 + c] = m.x0[n * 7 + c] + m.q[n * 7 + c];
        const V4 r = quat_compose(&m.q[n * 7 + 3], &m.x0[n * 7 + 3]);
        for (int c = 0; c < 4; ++c) m.x[n * 7 + 3 + c] = r[c];
    }
}

long find_offset(const orc_model& m, long row, long col) {
    const long* b = m.col_inds.data() + m.row_ptrs[row];
    const long* e = m.col_inds.data() + m.row_ptrs[row + 1];
    const long* p = std::lower_bound(b, e, col);
    return (p != e && *p == col) ? (p - m.col_inds.data()) : -1;
}

// src/system/beams/calculate_quadrature_point_values.hpp:51-172 for one element
void update_beam(orc_model& m, OBeam& B, double beta_prime, double gamma_prime) {
    const int N = B.N, Q = B.Q;
    std::vector<double> Fc(Q * 6), Fd(Q * 6), Fi(Q * 6), Fg(Q * 6);
    std::vector<double> Kuu(Q * 36), Puu(Q * 36), Cuu(Q * 36), Ouu(Q * 36), Quu(Q * 36),
        Muu(Q * 36), Guu(Q * 36);
#ifdef ORC_COUNT_FLOPS
    const long long qp_flops0 = g_flops;
#endif
    for (int qp = 0; qp < Q; ++qp) {
        // interpolate_to_quadrature_point_for_inertia.hpp:19-40
        double r[4] = {0, 0, 0, 0}, ud[3] = {0, 0, 0}, om[3] = {0, 0, 0}, omd[3] = {0, 0, 0};
        ORC_FLOPS(26 * N + 4);  // interpolation sums; the 4 divisions of the normalisation
        for (int n = 0; n < N; ++n) {
            const int s = B.node_ids[n];
            const double phi = B.phi[n * Q + qp];
            for (int c = 0; c < 3; ++c) {
                ud[c] += m.vd[s * 6 + c] * phi;
                om[c] += m.v[s * 6 + c + 3] * phi;
                omd[c] += m.vd[s * 6 + c + 3] * phi;
            }
            for (int c = 0; c < 4; ++c) r[c] += m.q[s * 7 + c + 3] * phi;
        }
        const double rl = nrm2(r, 4);
        for (int c = 0; c < 4; ++c) r[c] /= rl;
        inertial_qp(&B.mstar[qp * 36], &B.r0[qp * 4], r, ud, om, omd, m.gravity, &Fi[qp * 6],
                    &Fg[qp * 6], &Muu[qp * 36], &Guu[qp * 36], &Kuu[qp * 36]);
        // interpolate_to_quadrature_point_for_stiffness.hpp:19-41
        double u[3] = {0, 0, 0}, up[3] = {0, 0, 0}, r2[4] = {0, 0, 0, 0}, rp[4] = {0, 0, 0, 0};
        ORC_FLOPS(29 * N + 4);  // dphi / J and the interpolation sums; normalisation divisions
        for (int n = 0; n < N; ++n) {
            const int s = B.node_ids[n];
            const double phi = B.phi[n * Q + qp];
            const double dphiJ = B.dphi[n * Q + qp] / B.jac[qp];
            for (int c = 0; c < 3; ++c) {
                u[c] += m.q[s * 7 + c] * phi;
                up[c] += m.q[s * 7 + c] * dphiJ;
            }
            for (int c = 0; c < 4; ++c) {
                r2[c] += m.q[s * 7 + c + 3] * phi;
                rp[c] += m.q[s * 7 + c + 3] * dphiJ;
            }
        }
        const double rl2 = nrm2(r2, 4);
        for (int c = 0; c < 4; ++c) r2[c] /= rl2;
        stiffness_qp(&B.cstar[qp * 36], &B.r0[qp * 4], &B.x0p[qp * 3], up, r2, rp, &Fc[qp * 6],
                     &Fd[qp * 6], &Cuu[qp * 36], &Ouu[qp * 36], &Puu[qp * 36], &Quu[qp * 36]);
    }
#ifdef ORC_COUNT_FLOPS
    g_qp_flops += g_flops - qp_flops0;
#endif
    std::vector<double> S(N * N * 36), I(N * N * 36);
    if (m.solver_mode & 2) {
        // Cross-check ordering: the same sums with the quadrature points reversed.
        auto rev = [Q](const std::vector<double>& a, int w) {
            std::vector<double> r(a.size());
            for (int q = 0; q < Q; ++q)
                for (int k = 0; k < w; ++k) r[(Q - 1 - q) * w + k] = a[q * w + k];
            return r;
        };
        auto revn = [N, Q](const std::vector<double>& a) {
            std::vector<double> r(a.size());
            for (int n = 0; n < N; ++n)
                for (int q = 0; q < Q; ++q) r[n * Q + (Q - 1 - q)] = a[n * Q + q];
            return r;
        };
        const auto w = rev(B.w, 1), jac = rev(B.jac, 1), phi = revn(B.phi), dphi = revn(B.dphi);
        orc_integrate_residual(N, Q, w.data(), jac.data(), phi.data(), dphi.data(), B.fx.data(),
                               rev(Fc, 6).data(), rev(Fd, 6).data(), rev(Fi, 6).data(),
                               B.fe.data(), rev(Fg, 6).data(), B.residual.data());
        orc_integrate_stiffness(N, Q, w.data(), jac.data(), phi.data(), dphi.data(),
                                rev(Kuu, 36).data(), rev(Puu, 36).data(), rev(Cuu, 36).data(),
                                rev(Ouu, 36).data(), rev(Quu, 36).data(), S.data());
        orc_integrate_inertia(N, Q, w.data(), jac.data(), phi.data(), rev(Muu, 36).data(),
                              rev(Guu, 36).data(), beta_prime, gamma_prime, I.data());
    } else {
        orc_integrate_residual(N, Q, B.w.data(), B.jac.data(), B.phi.data(), B.dphi.data(),
                               B.fx.data(), Fc.data(), Fd.data(), Fi.data(), B.fe.data(),
                               Fg.data(), B.residual.data());
        orc_integrate_stiffness(N, Q, B.w.data(), B.jac.data(), B.phi.data(), B.dphi.data(),
                                Kuu.data(), Puu.data(), Cuu.data(), Ouu.data(), Quu.data(),
                                S.data());
        orc_integrate_inertia(N, Q, B.w.data(), B.jac.data(), B.phi.data(), Muu.data(),
                              Guu.data(), beta_prime, gamma_prime, I.data());
    }
    // calculate_system_matrix.hpp:25-53
    for (int i = 0; i < N; ++i) {
        for (int j = 0; j < N; ++j) {
            const int nT = B.node_ids[j];
            double* out = &B.sysmat[(i * N + j) * 36];
            for (int k = 0; k < 36; ++k) out[k] = I[(i * N + j) * 36 + k];
            gemm(false, false, 6, 6, 6, 1., &S[(i * N + j) * 36], 6, &m.tangent[nT * 36], 6, 1.,
                 out, 6);
        }
    }
}

// src/system/masses/calculate_quadrature_point_values.hpp:40-152 (one mass at its
// node: vd as the acceleration, residual Fi - Fg, matrix b'Muu + g'Guu + Kuu T)
void update_mass(orc_model& m, OMass& M, double beta_prime, double gamma_prime) {
    const int n = M.node;
    const double* q = &m.q[n * 7];
    const double* v = &m.v[n * 6];
    const double* vd = &m.vd[n * 6];
    double FI[6], FG[6], Muu[36], Guu[36], Kuu[36];
    inertial_qp(M.mstar, M.r0, q + 3, vd, v + 3, vd + 3, m.gravity, FI, FG, Muu, Guu, Kuu);
    for (int c = 0; c < 6; ++c) M.residual[c] = FI[c] - FG[c];
    for (int k = 0; k < 36; ++k) M.sysmat[k] = beta_prime * Muu[k] + gamma_prime * Guu[k];
    gemm(false, false, 6, 6, 6, 1., Kuu, 6, &m.tangent[n * 36], 6, 1., M.sysmat, 6);
}

// src/system/springs/calculate_quadrature_point_values.hpp:27-92 with
// calculate_{distance_components,length,force_coefficients,force_vectors,stiffness_matrix}.hpp
void update_spring(orc_model& m, OSpring& S) {
    const double* u1 = &m.q[S.n1 * 7];
    const double* u2 = &m.q[S.n2 * 7];
    double r[3];
    for (int c = 0; c < 3; ++c) r[c] = S.x0[c] + u2[c] - u1[c];
    const double l = std::sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
    const double c1 = S.k * (S.l_ref / l - 1.);
    const double c2 = S.k * S.l_ref / (l * l * l);
    double f[3];
    for (int c = 0; c < 3; ++c) f[c] = c1 * r[c];
    double a[9] = {};
    const double diag = c1 - c2 * l * l;
    a[0] = a[4] = a[8] = diag;
    const M3 rt = tilde(r);
    gemm(false, false, 3, 3, 3, -c2, rt.data(), 3, rt.data(), 3, 1., a, 3);
    for (int c = 0; c < 3; ++c) {
        S.residual[0][c] = f[c];
        S.residual[1][c] = -f[c];
    }
    for (int k = 0; k < 9; ++k) {
        S.stiff[0][0][k] = a[k];
        S.stiff[0][1][k] = -a[k];
        S.stiff[1][0][k] = -a[k];
        S.stiff[1][1][k] = a[k];
    }
}

// src/constraints/calculate_constraint_residual_gradient.hpp:60-199 (FixedBC, PrescribedBC)
void update_rigid_joint(orc_model& m, OConstraint& C);
void update_revolute_joint(orc_model& m, OConstraint& C);
void update_3dof_constraint(orc_model& m, OConstraint& C);

void update_constraint(orc_model& m, OConstraint& C) {
    if (C.type == KYN_CONSTRAINT_RIGID_JOINT || C.type == KYN_CONSTRAINT_ROTATION_CONTROL) {
        update_rigid_joint(m, C);
        return;
    }
    if (C.type == KYN_CONSTRAINT_REVOLUTE_JOINT) {
        update_revolute_joint(m, C);
        return;
    }
    if (C.type >= KYN_CONSTRAINT_FIXED_BC_3DOF) {
        update_3dof_constraint(m, C);
        return;
    }
    const double* nu = &m.q[C.target * 7];
    double u1[3] = {0., 0., 0.};
    double R1[4] = {1., 0., 0., 0.};
    if (C.type == KYN_CONSTRAINT_PRESCRIBED_BC) {
        for (int i = 0; i < 3; ++i) u1[i] = C.input[i];
        for (int i = 0; i < 4; ++i) R1[i] = C.input[3 + i];
    }
    const double u2[3] = {nu[0], nu[1], nu[2]};
    const double R2[4] = {nu[3], nu[4], nu[5], nu[6]};
    const V4 R1t = quat_inverse(R1);
    const V3 R1X0 = rotate_vec(R1, C.X0);
    for (int c = 0; c < 3; ++c) C.res[c] = u2[c] + C.X0[c] - u1[c] - R1X0[c];
    const V4 R2R1t = quat_compose(R2, R1t.data());
    const M3 Cm = quat_to_rot(R2R1t.data());
    const V3 ax = axial(Cm);
    for (int c = 0; c < 3; ++c) C.res[3 + c] = ax[c];
    M6 grad{};
    for (int c = 0; c < 3; ++c) grad[c * 7] = 1.;
    const M3 A = ax_matrix(Cm);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) grad[(3 + i) * 6 + 3 + j] = A[j * 3 + i];
    for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j) C.t_grad_trans[i * 6 + j] = grad[j * 6 + i];
    gemm(false, false, 6, 6, 6, 1., grad.data(), 6, &m.tangent[C.target * 36], 6, 0.,
         C.t_grad_tan, 6);
    gemv(false, 6, 6, 1., C.t_grad_trans, 6, C.lambda, 0., C.t_lambda_res);
}

// src/constraints/calculate_rigid_joint_constraint.hpp:17-113 and the RigidJoint
// branch of calculate_constraint_residual_gradient.hpp:251-320.  RotationControl
// (calculate_rotation_control_constraint.hpp:17-144, branch :468-540) is the same
// joint with the commanded rotation Rc = exp(input[0] axis) in the rotational
// residual: C = R(R2 Rc^-1 R1^-1).
void update_rigid_joint(orc_model& m, OConstraint& C) {
    const double* bu = &m.q[C.base * 7];
    const double* tu = &m.q[C.target * 7];
    const double u1[3] = {bu[0], bu[1], bu[2]};
    const double R1[4] = {bu[3], bu[4], bu[5], bu[6]};
    const double u2[3] = {tu[0], tu[1], tu[2]};
    const double R2[4] = {tu[3], tu[4], tu[5], tu[6]};
    const V4 R1t = quat_inverse(R1);
    const V3 R1X0 = rotate_vec(R1, C.X0);
    for (int c = 0; c < 3; ++c) C.res[c] = u2[c] + C.X0[c] - u1[c] - R1X0[c];
    V4 R2R1t;
    if (C.type == KYN_CONSTRAINT_ROTATION_CONTROL) {
        const double rv[3] = {C.axis[0] * C.input[0], C.axis[1] * C.input[0], C.axis[2] * C.input[0]};
        const V4 Rc = rotvec_to_quat(rv);
        const V4 Rct = quat_inverse(Rc.data());
        const V4 R2Rct = quat_compose(R2, Rct.data());
        R2R1t = quat_compose(R2Rct.data(), R1t.data());
    } else {
        R2R1t = quat_compose(R2, R1t.data());
    }
    const M3 Cm = quat_to_rot(R2R1t.data());
    const V3 ax = axial(Cm);
    for (int c = 0; c < 3; ++c) C.res[3 + c] = ax[c];
    const M3 A = ax_matrix(Cm);
    M6 tg{}, bg{};
    for (int c = 0; c < 3; ++c) tg[c * 7] = 1.;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) tg[(3 + i) * 6 + 3 + j] = A[j * 3 + i];
    for (int c = 0; c < 3; ++c) bg[c * 7] = -1.;
    // B(0:3,3:6) = tilde(R1 X0)
    const double tl[9] = {0., -R1X0[2], R1X0[1], R1X0[2], 0., -R1X0[0], -R1X0[1], R1X0[0], 0.};
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) bg[i * 6 + 3 + j] = tl[i * 3 + j];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) bg[(3 + i) * 6 + 3 + j] = -A[i * 3 + j];
    for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j) {
            C.t_grad_trans[i * 6 + j] = tg[j * 6 + i];
            C.b_grad_trans[i * 6 + j] = bg[j * 6 + i];
        }
    gemm(false, false, 6, 6, 6, 1., bg.data(), 6, &m.tangent[C.base * 36], 6, 0., C.b_grad_tan, 6);
    gemm(false, false, 6, 6, 6, 1., tg.data(), 6, &m.tangent[C.target * 36], 6, 0., C.t_grad_tan, 6);
    gemv(false, 6, 6, 1., C.b_grad_trans, 6, C.lambda, 0., C.b_lambda_res);
    gemv(false, 6, 6, 1., C.t_grad_trans, 6, C.lambda, 0., C.t_lambda_res);
}

// src/constraints/calculate_revolute_joint_constraint.hpp:19-113 and
// calculate_revolute_joint_force.hpp:19-45 with the RevoluteJoint branch of
// calculate_constraint_residual_gradient.hpp:388-465.  Five rows: the relative
// translation, and the two dot products (R2 z0).(R1 x0), (R2 y0).(R1 x0) that
// vanish while the target's frame keeps the joint axis; row 5 of the 6x6
// blocks stays zero.  The torque input[0] about R2 x0 joins the target's rows.
void update_revolute_joint(orc_model& m, OConstraint& C) {
    const double* bu = &m.q[C.base * 7];
    const double* tu = &m.q[C.target * 7];
    const double* x0 = C.axes;
    const double* y0 = C.axes + 3;
    const double* z0 = C.axes + 6;
    const double R1[4] = {bu[3], bu[4], bu[5], bu[6]};
    const double R2[4] = {tu[3], tu[4], tu[5], tu[6]};
    const V3 R1X0 = rotate_vec(R1, C.X0);
    for (int c = 0; c < 3; ++c) C.res[c] = tu[c] + C.X0[c] - bu[c] - R1X0[c];
    const V3 x = rotate_vec(R1, x0);
    const V3 y = rotate_vec(R2, y0);
    const V3 z = rotate_vec(R2, z0);
    C.res[3] = z[0] * x[0] + z[1] * x[1] + z[2] * x[2];
    C.res[4] = y[0] * x[0] + y[1] * x[1] + y[2] * x[2];
    C.res[5] = 0.;
    const double xcz[3] = {x[1] * z[2] - x[2] * z[1], x[2] * z[0] - x[0] * z[2], x[0] * z[1] - x[1] * z[0]};
    const double xcy[3] = {x[1] * y[2] - x[2] * y[1], x[2] * y[0] - x[0] * y[2], x[0] * y[1] - x[1] * y[0]};
    M6 tg{}, bg{};
    for (int c = 0; c < 3; ++c) {
        tg[c * 7] = 1.;
        bg[c * 7] = -1.;
        tg[3 * 6 + 3 + c] = -xcz[c];
        tg[4 * 6 + 3 + c] = -xcy[c];
        bg[3 * 6 + 3 + c] = xcz[c];
        bg[4 * 6 + 3 + c] = xcy[c];
    }
    for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j) {
            C.t_grad_trans[i * 6 + j] = tg[j * 6 + i];
            C.b_grad_trans[i * 6 + j] = bg[j * 6 + i];
        }
    gemm(false, false, 6, 6, 6, 1., bg.data(), 6, &m.tangent[C.base * 36], 6, 0., C.b_grad_tan, 6);
    gemm(false, false, 6, 6, 6, 1., tg.data(), 6, &m.tangent[C.target * 36], 6, 0., C.t_grad_tan, 6);
    gemv(false, 6, 6, 1., C.b_grad_trans, 6, C.lambda, 0., C.b_lambda_res);
    gemv(false, 6, 6, 1., C.t_grad_trans, 6, C.lambda, 0., C.t_lambda_res);
    const V3 ax = rotate_vec(R2, x0);
    for (int c = 0; c < 3; ++c) {
        C.sys_res[c] = 0.;
        C.sys_res[3 + c] = ax[c] * C.input[0];
    }
}

// Three-row constraints on a position-only target
// (calculate_fixed_bc_3DOF_constraint.hpp, calculate_prescribed_bc_3DOF_constraint.hpp,
// calculate_rigid_joint_3DOF_constraint.hpp with their branches of
// calculate_constraint_residual_gradient.hpp:101-150, 196-248): residual
// u2 + X0 - u1 - R1 X0 (FixedBC: u1 = 0, R1 = I; PrescribedBC: (u1, R1) = the
// input; joint: the base node's displacement), target gradient I on the
// translation, joint base gradient [-I, tilde(R1 X0)].
void update_3dof_constraint(orc_model& m, OConstraint& C) {
    const double* tu = &m.q[C.target * 7];
    double u1[3] = {0., 0., 0.};
    double R1[4] = {1., 0., 0., 0.};
    if (C.type == KYN_CONSTRAINT_PRESCRIBED_BC_3DOF) {
        for (int i = 0; i < 3; ++i) u1[i] = C.input[i];
        for (int i = 0; i < 4; ++i) R1[i] = C.input[3 + i];
    } else if (C.type == KYN_CONSTRAINT_RIGID_JOINT_6DOF_TO_3DOF) {
        const double* bu = &m.q[C.base * 7];
        for (int i = 0; i < 3; ++i) u1[i] = bu[i];
        for (int i = 0; i < 4; ++i) R1[i] = bu[3 + i];
    }
    const V3 R1X0 = rotate_vec(R1, C.X0);
    for (int c = 0; c < 3; ++c) C.res[c] = tu[c] + C.X0[c] - u1[c] - R1X0[c];
    for (int c = 3; c < 6; ++c) C.res[c] = 0.;
    M6 tg{}, bg{};
    for (int c = 0; c < 3; ++c) tg[c * 7] = 1.;
    if (C.type == KYN_CONSTRAINT_RIGID_JOINT_6DOF_TO_3DOF) {
        for (int c = 0; c < 3; ++c) bg[c * 7] = -1.;
        const double tl[9] = {0., -R1X0[2], R1X0[1], R1X0[2], 0., -R1X0[0], -R1X0[1], R1X0[0], 0.};
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) bg[i * 6 + 3 + j] = tl[i * 3 + j];
    }
    for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j) {
            C.t_grad_trans[i * 6 + j] = tg[j * 6 + i];
            C.b_grad_trans[i * 6 + j] = bg[j * 6 + i];
        }
    gemm(false, false, 6, 6, 6, 1., tg.data(), 6, &m.tangent[C.target * 36], 6, 0., C.t_grad_tan, 6);
    gemv(false, 6, 6, 1., C.t_grad_trans, 6, C.lambda, 0., C.t_lambda_res);
    if (C.type == KYN_CONSTRAINT_RIGID_JOINT_6DOF_TO_3DOF) {
        gemm(false, false, 6, 6, 6, 1., bg.data(), 6, &m.tangent[C.base * 36], 6, 0., C.b_grad_tan, 6);
        gemv(false, 6, 6, 1., C.b_grad_trans, 6, C.lambda, 0., C.b_lambda_res);
    }
}

// src/constraints/calculate_revolute_joint_output.hpp:24-85: rotation about
// the joint axis (axis turned by the target's rotation, dotted with the
// rotation vector of that rotation), angular velocity and acceleration about
// it.
void revolute_output(const orc_model& m, OConstraint& C) {
    const double* u = &m.q[C.target * 7];
    const double R[4] = {u[3], u[4], u[5], u[6]};
    const V3 ax = rotate_vec(R, C.axes);
    double rv[3] = {0., 0., 0.};
    const double s = std::sqrt(1. - R[0] * R[0]);
    if (s > 1e-12) {  // src/math/quaternion_operations.hpp QuaternionToRotationVector
        const double th = 2. * std::acos(R[0]);
        for (int c = 0; c < 3; ++c) rv[c] = th * R[1 + c] / s;
    }
    const double* w = &m.v[C.target * 6 + 3];
    const double* wd = &m.vd[C.target * 6 + 3];
    C.output[0] = ax[0] * rv[0] + ax[1] * rv[1] + ax[2] * rv[2];
    C.output[1] = ax[0] * w[0] + ax[1] * w[1] + ax[2] * w[2];
    C.output[2] = ax[0] * wd[0] + ax[1] * wd[1] + ax[2] * wd[2];
}

// Solver of the oracle (bit flags of orc_model::solver_mode): 0 = dense LU
// with partial pivoting of the whole bordered system (default); bit 1 =
// elimination of the single-node boundary conditions followed by LU without
// pivoting of the free block; bit 2 = quadrature sums taken in reverse order.
// The flagged variants are the same FP64 algorithm in another summation order;
// their distance from the default measures the rounding-noise floor.
void solve_eliminated(orc_model& m);

void solve_dense(orc_model& m) {
    bool special = false;  // rows the single-node elimination does not cover
    for (auto& C : m.cons)
        special = special || C.type == KYN_CONSTRAINT_REVOLUTE_JOINT || C.type >= KYN_CONSTRAINT_FIXED_BC_3DOF;
    if ((m.solver_mode & 1) && !special) {
        solve_eliminated(m);
        return;
    }
    // Dense LU with partial pivoting of the CRS system A x = b.
    const long n = m.ndofs;
    std::vector<double> A(n * n, 0.);
    for (long r = 0; r < n; ++r)
        for (long k = m.row_ptrs[r]; k < m.row_ptrs[r + 1]; ++k) A[r * n + m.col_inds[k]] = m.values[k];
    std::vector<double> x(m.b);
    std::vector<long> piv(n);
    for (long k = 0; k < n; ++k) {
        long p = k;
        double best = std::abs(A[k * n + k]);
        for (long i = k + 1; i < n; ++i) {
            if (std::abs(A[i * n + k]) > best) {
                best = std::abs(A[i * n + k]);
                p = i;
            }
        }
        if (p != k) {
            for (long j = 0; j < n; ++j) std::swap(A[k * n + j], A[p * n + j]);
            std::swap(x[k], x[p]);
        }
        const double d = A[k * n + k];
        for (long i = k + 1; i < n; ++i) {
            const double l = A[i * n + k] / d;
            A[i * n + k] = l;
            if (l == 0.) continue;
            for (long j = k + 1; j < n; ++j) A[i * n + j] -= l * A[k * n + j];
            x[i] -= l * x[k];
        }
    }
    for (long i = n - 1; i >= 0; --i) {
        double s = x[i];
        for (long j = i + 1; j < n; ++j) s -= A[i * n + j] * x[j];
        x[i] = s / A[i * n + i];
    }
    m.xsol = x;
}

void solve_eliminated(orc_model& m) {
    const long n = m.ndofs;
    std::vector<double> A(n * n, 0.);
    for (long r = 0; r < n; ++r)
        for (long k = m.row_ptrs[r]; k < m.row_ptrs[r + 1]; ++k) A[r * n + m.col_inds[k]] = m.values[k];
    std::vector<char> constrained(m.nsys, 0);
    for (auto& C : m.cons)
        for (int c = 0; c < 6; ++c) constrained[C.target_table[c]] = 1;
    std::vector<long> fr;
    for (long i = 0; i < m.nsys; ++i)
        if (!constrained[i]) fr.push_back(i);
    std::vector<double> x(n, 0.);
    // B x_r = b_lambda for each constraint (6x6 dense solve with pivoting)
    for (auto& C : m.cons) {
        double M[6][7];
        for (int i = 0; i < 6; ++i) {
            for (int j = 0; j < 6; ++j) M[i][j] = A[(m.nsys + C.row_first + i) * n + C.target_table[j]];
            M[i][6] = m.b[m.nsys + C.row_first + i];
        }
        for (int k = 0; k < 6; ++k) {
            int p = k;
            for (int i = k + 1; i < 6; ++i) if (std::abs(M[i][k]) > std::abs(M[p][k])) p = i;
            for (int j = 0; j < 7; ++j) std::swap(M[k][j], M[p][j]);
            for (int i = k + 1; i < 6; ++i) {
                const double l = M[i][k] / M[k][k];
                for (int j = k; j < 7; ++j) M[i][j] -= l * M[k][j];
            }
        }
        for (int i = 5; i >= 0; --i) {
            double s2 = M[i][6];
            for (int j = i + 1; j < 6; ++j) s2 -= M[i][j] * x[C.target_table[j]];
            x[C.target_table[i]] = s2 / M[i][i];
        }
    }
    const long mf = static_cast<long>(fr.size());
    std::vector<double> F(mf * mf), y(mf);
    for (long a = 0; a < mf; ++a) {
        double r = m.b[fr[a]];
        for (long j = 0; j < m.nsys; ++j) if (constrained[j]) r -= A[fr[a] * n + j] * x[j];
        y[a] = r;
        for (long c = 0; c < mf; ++c) F[a * mf + c] = A[fr[a] * n + fr[c]];
    }
    for (long k = 0; k < mf; ++k) {
        const double rp = 1. / F[k * mf + k];
        for (long i = k + 1; i < mf; ++i) {
            const double l = F[i * mf + k] * rp;
            for (long j = k + 1; j < mf; ++j) F[i * mf + j] -= l * F[k * mf + j];
            y[i] -= l * y[k];
        }
    }
    for (long i = mf - 1; i >= 0; --i) {
        double s2 = y[i];
        for (long j = i + 1; j < mf; ++j) s2 -= F[i * mf + j] * x[fr[j]];
        x[fr[i]] = s2 / F[i * mf + i];
    }
    // multipliers from the constrained rows: G^T x_lambda = b_r - A_r x
    for (auto& C : m.cons) {
        double M[6][7];
        for (int i = 0; i < 6; ++i) {
            const long row = C.target_table[i];
            double r = m.b[row];
            for (long j = 0; j < m.nsys; ++j) r -= A[row * n + j] * x[j];
            for (int j = 0; j < 6; ++j) M[i][j] = A[row * n + m.nsys + C.row_first + j];
            M[i][6] = r;
        }
        for (int k = 0; k < 6; ++k) {
            int p = k;
            for (int i = k + 1; i < 6; ++i) if (std::abs(M[i][k]) > std::abs(M[p][k])) p = i;
            for (int j = 0; j < 7; ++j) std::swap(M[k][j], M[p][j]);
            for (int i = k + 1; i < 6; ++i) {
                const double l = M[i][k] / M[k][k];
                for (int j = k; j < 7; ++j) M[i][j] -= l * M[k][j];
            }
        }
        for (int i = 5; i >= 0; --i) {
            double s2 = M[i][6];
            for (int j = i + 1; j < 6; ++j) s2 -= M[i][j] * x[m.nsys + C.row_first + j];
            x[m.nsys + C.row_first + i] = s2 / M[i][i];
        }
    }
    m.xsol = x;
}

struct Params {
    bool dynamic;
    int max_iter;
    double h, am, af, gamma, beta, gp, bp, cond, atol, rtol;
};

// src/step/step_parameters.hpp:37-52
Params make_params(const kyn_step_params* p) {
    Params q{};
    q.dynamic = p->is_dynamic_solve != 0;
    q.max_iter = p->max_iter;
    q.h = p->h;
    const double rho = p->rho_inf;
    q.am = (2. * rho - 1.) / (rho + 1.);
    q.af = rho / (rho + 1.);
    q.gamma = 0.5 + q.af - q.am;
    q.beta = 0.25 * (q.gamma + 0.5) * (q.gamma + 0.5);
    q.gp = q.dynamic ? q.gamma / (q.h * q.beta) : 0.;
    q.bp = q.dynamic ? (1. - q.am) / (q.h * q.h * q.beta * (1. - q.af)) : 0.;
    q.cond = q.beta * q.h * q.h;
    q.atol = p->absolute_convergence_tol;
    q.rtol = p->relative_convergence_tol;
    return q;
}

// src/step/predict_next_state.hpp:14-47
void predict(orc_model& m, const Params& P) {
    m.q_prev = m.q;
    calculate_next_state(m, P.h, P.af, P.am, P.beta, P.gamma);
    calculate_displacement(m, P.h);
}

void assemble(orc_model& m, const Params& P) {
    // src/step/reset_solver.hpp
    std::fill(m.values.begin(), m.values.end(), 0.);
    std::fill(m.b.begin(), m.b.end(), 0.);
    // src/step/update_tangent_operator.hpp
    for (int n = 0; n < m.num_nodes; ++n) tangent_operator(P.h, &m.q_delta[n * 6], &m.tangent[n * 36]);
    // src/step/update_system_variables_beams.hpp
    for (auto& B : m.beams) update_beam(m, B, P.bp, P.gp);
    // src/step/update_system_variables.hpp:23-28 (masses, springs)
    for (auto& M : m.masses) update_mass(m, M, P.bp, P.gp);
    for (auto& S : m.springs) update_spring(m, S);
    // src/step/assemble_system_residual.hpp:17-64 (forces, beams, masses, springs)
    for (int n = 0; n < m.num_nodes; ++n) {
        const long d = m.fmap[n];
        const unsigned s = m.sig[n];
        if (s == 0b111111U) {
            for (int c = 0; c < 6; ++c) m.b[d + c] -= m.f[n * 6 + c];
        } else if (s == 0b111000U) {
            for (int c = 0; c < 3; ++c) m.b[d + c] -= m.f[n * 6 + c];
        } else if (s == 0b000111U) {
            for (int c = 0; c < 3; ++c) m.b[d + c] -= m.f[n * 6 + 3 + c];
        }
    }
    for (auto& B : m.beams)
        for (int n = 0; n < B.N; ++n)
            for (int c = 0; c < 6; ++c) m.b[B.eft[n * 6 + c]] += B.residual[n * 6 + c];
    for (auto& M : m.masses)  // src/solver/contribute_masses_to_vector.hpp
        for (int c = 0; c < 6; ++c) m.b[M.eft[c]] += M.residual[c];
    for (auto& S : m.springs)  // src/solver/contribute_springs_to_vector.hpp
        for (int c = 0; c < 3; ++c) {
            m.b[S.eft[0][c]] += S.residual[0][c];
            m.b[S.eft[1][c]] += S.residual[1][c];
        }
    // src/step/assemble_system_matrix.hpp -> contribute_beams_to_sparse_matrix.hpp:34-73
    for (auto& B : m.beams) {
        for (int n2 = 0; n2 < B.N; ++n2) {
            for (int n1 = 0; n1 < B.N; ++n1) {
                const long first_col = B.eft[n2 * 6];
                for (int c1 = 0; c1 < 6; ++c1) {
                    const long row = B.eft[n1 * 6 + c1];
                    long off = find_offset(m, row, first_col);
                    for (int c2 = 0; c2 < 6; ++c2, ++off)
                        m.values[off] += B.sysmat[(n1 * B.N + n2) * 36 + c1 * 6 + c2] * P.cond;
                }
            }
        }
    }
    // src/solver/contribute_masses_to_sparse_matrix.hpp
    for (auto& M : m.masses) {
        for (int c1 = 0; c1 < 6; ++c1) {
            long off = find_offset(m, M.eft[c1], M.eft[0]);
            for (int c2 = 0; c2 < 6; ++c2, ++off) m.values[off] += M.sysmat[c1 * 6 + c2] * P.cond;
        }
    }
    // src/solver/contribute_springs_to_sparse_matrix.hpp
    for (auto& S : m.springs) {
        for (int a = 0; a < 2; ++a)
            for (int b = 0; b < 2; ++b)
                for (int c1 = 0; c1 < 3; ++c1) {
                    long off = find_offset(m, S.eft[a][c1], S.eft[b][0]);
                    for (int c2 = 0; c2 < 3; ++c2, ++off)
                        m.values[off] += S.stiff[a][b][c1 * 3 + c2] * P.cond;
                }
    }
    // src/step/update_constraint_variables.hpp
    for (auto& C : m.cons) update_constraint(m, C);
    // src/step/assemble_constraints_matrix.hpp
    for (auto& C : m.cons) {
        for (long i = C.row_first; i < C.row_last; ++i) {
            const long rn = i - C.row_first;
            const long row = m.nsys + i;
            if (C.base_active) {  // src/solver/copy_constraints_to_sparse_matrix.hpp:37-84
                long boff = find_offset(m, row, C.base_table[0]);
                for (long e = 0; e < C.base_active; ++e, ++boff) m.values[boff] += C.b_grad_tan[rn * 6 + e];
            }
            long off = find_offset(m, row, C.target_table[0]);
            for (long e = 0; e < C.target_active; ++e, ++off) m.values[off] += C.t_grad_tan[rn * 6 + e];
        }
        const long first_col = C.row_first + m.nsys;
        const long ncols = C.row_last - C.row_first;
        for (long i = C.base_table[0]; C.base_active && i < C.base_table[0] + C.base_active; ++i) {
            const long rn = i - C.base_table[0];
            long off = find_offset(m, i, first_col);
            for (long e = 0; e < ncols; ++e, ++off) m.values[off] += C.b_grad_trans[rn * 6 + e];
        }
        for (long i = C.target_table[0]; i < C.target_table[0] + C.target_active; ++i) {
            const long rn = i - C.target_table[0];
            long off = find_offset(m, i, first_col);
            for (long e = 0; e < ncols; ++e, ++off) m.values[off] += C.t_grad_trans[rn * 6 + e];
        }
    }
    // src/step/assemble_constraints_residual.hpp
    for (auto& C : m.cons)
        for (long c = 0; c < C.target_active; ++c) m.b[C.target_table[c]] += C.sys_res[c];
    for (auto& C : m.cons)  // src/solver/contribute_lambda_to_vector.hpp:34-51
        for (long c = 0; c < C.base_active; ++c) m.b[C.base_table[0] + c] += C.b_lambda_res[c];
    for (auto& C : m.cons)
        for (long c = 0; c < C.target_active; ++c) m.b[C.target_table[0] + c] += C.t_lambda_res[c];
    for (auto& C : m.cons)
        for (long c = 0; c < C.row_last - C.row_first; ++c) m.b[m.nsys + C.row_first + c] += C.res[c];
}

// src/step/step.hpp:42-124
int step_impl(orc_model& m, const Params& P, int* iters) {
    predict(m, P);
    // src/step/reset_constraints.hpp
    for (auto& C : m.cons) {
        for (int c = 0; c < 6; ++c) {
            C.lambda[c] = 0.;
            C.sys_res[c] = 0.;
        }
    }
    m.conv.clear();
    double err = 1000.;
    for (int iter = 0; err > 1.; ++iter) {
        if (iter >= P.max_iter) {
            if (iters) *iters = iter;
            return KYN_NOT_CONVERGED;
        }
        assemble(m, P);
        // src/step/solve_system.hpp:15-39
        for (long i = 0; i < m.nsys; ++i) m.b[i] *= P.cond;
        for (long i = 0; i < m.ndofs; ++i) m.b[i] = -1. * m.b[i];
        solve_dense(m);
        for (long i = m.nsys; i < m.ndofs; ++i) m.xsol[i] /= P.cond;
        // src/step/calculate_convergence_error.hpp:16-54
        double sum_sys = 0.;
        for (int n = 0; n < m.num_nodes; ++n) {
            for (long c = 0; c < m.active[n]; ++c) {
                const double pi = m.xsol[m.fmap[n] + c];
                const double xi = m.q_delta[n * 6 + c] * P.h;
                const double e = pi / (P.atol + P.rtol * std::abs(xi));
                sum_sys += e * e;
            }
        }
        double sum_con = 0.;
        for (auto& C : m.cons) {
            for (long r = C.row_first; r < C.row_last; ++r) {
                const double pi = m.xsol[m.nsys + r];
                const double xi = C.lambda[r - C.row_first];
                const double e = pi / (P.atol + P.rtol * std::abs(xi));
                sum_con += e * e;
            }
        }
        err = std::sqrt((sum_sys + sum_con) / static_cast<double>(m.ndofs));
        m.conv.push_back(err);
        // src/step/update_state_prediction.hpp
        for (int n = 0; n < m.num_nodes; ++n) {
            const int nd = count_bits(m.sig[n]);
            const long fd = m.fmap[n];
            for (int c = 0; c < nd; ++c) {
                const double delta = m.xsol[fd + c];
                m.q_delta[n * 6 + c] += delta / P.h;
                if (P.dynamic) {
                    m.v[n * 6 + c] += P.gp * delta;
                    m.vd[n * 6 + c] += P.bp * delta;
                }
            }
        }
        calculate_displacement(m, P.h);
        // src/constraints/update_lambda_prediction.hpp:27-42
        for (auto& C : m.cons)
            for (long r = C.row_first; r < C.row_last; ++r)
                C.lambda[r - C.row_first] += m.xsol[m.nsys + r];
    }
    // src/state/update_algorithmic_acceleration.hpp:19-23, update_global_position.hpp
    for (int n = 0; n < m.num_nodes; ++n)
        for (int c = 0; c < 6; ++c) m.a[n * 6 + c] += (1. - P.af) / (1. - P.am) * m.vd[n * 6 + c];
    update_global_position(m);
    // src/step/step.hpp:105-115 (CalculateConstraintOutput)
    for (auto& C : m.cons)
        if (C.type == KYN_CONSTRAINT_REVOLUTE_JOINT) revolute_output(m, C);
    if (iters) *iters = static_cast<int>(m.conv.size());
    return KYN_OK;
}

bool bad(char* err, int errlen, const char* msg) {
    if (err && errlen > 0) std::snprintf(err, static_cast<size_t>(errlen), "%s", msg);
    return false;
}

}  // namespace

extern "C" {

long orc_crs_build(int num_system_dofs, int num_dofs, int num_nodes, const long* active_dofs,
                   const long* fmap, int num_elems, int max_nodes, const long* nodes_per_elem,
                   const long* elem_nodes, int num_constraints, const long* base_active,
                   const long* target_active, const long* base_table, const long* target_table,
                   const long* row_range, long* row_ptrs, long* col_inds, int sort_rows) {
    // src/solver/compute_system_row_entries.hpp:75-102
    auto elem_contains = [&](int e, long node) {
        for (long k = 0; k < nodes_per_elem[e]; ++k)
            if (elem_nodes[e * max_nodes + k] == node) return true;
        return false;
    };
    auto con_contains = [&](int c, long dof) {
        const bool b = dof == base_table[c * 6] && base_active[c] != 0;
        const bool t = dof == target_table[c * 6] && target_active[c] != 0;
        return b || t;
    };
    std::vector<long> entries(num_dofs, 0);
    for (long node = 0; node < num_nodes; ++node) {
        const long nd = active_dofs[node];
        const long di = fmap[node];
        long e_row = nd;
        for (int e = 0; e < num_elems; ++e) {
            if (!elem_contains(e, node)) continue;
            long ent = 0;
            for (long k = 0; k < nodes_per_elem[e]; ++k) ent += active_dofs[elem_nodes[e * max_nodes + k]];
            e_row += ent - nd;
        }
        for (int c = 0; c < num_constraints; ++c) {
            if (!con_contains(c, di)) continue;
            e_row += row_range[c * 2 + 1] - row_range[c * 2];
        }
        for (long k = 0; k < nd; ++k) entries[di + k] = e_row;
    }
    // src/solver/compute_constraints_row_entries.hpp:26-34
    for (int c = 0; c < num_constraints; ++c)
        for (long r = row_range[c * 2]; r < row_range[c * 2 + 1]; ++r)
            entries[r + num_system_dofs] = base_active[c] + target_active[c];
    // src/solver/scan_row_entries.hpp
    std::vector<long> rp(num_dofs + 1, 0);
    for (int i = 0; i < num_dofs; ++i) rp[i + 1] = rp[i] + entries[i];
    if (row_ptrs) std::copy(rp.begin(), rp.end(), row_ptrs);
    const long nnz = rp[num_dofs];
    if (!col_inds) return nnz;
    // src/solver/compute_system_col_inds.hpp:91-131
    for (long node = 0; node < num_nodes; ++node) {
        const long nd = active_dofs[node];
        const long di = fmap[node];
        long cur[6] = {0, 0, 0, 0, 0, 0};
        for (long c1 = 0; c1 < nd; ++c1) {
            long idx = rp[di + c1];
            for (long c2 = 0; c2 < nd; ++c2, ++idx) col_inds[idx] = di + c2;
            cur[c1] = nd;
        }
        for (int e = 0; e < num_elems; ++e) {
            if (!elem_contains(e, node)) continue;
            for (long c = 0; c < nd; ++c) {
                long idx = rp[di + c] + cur[c];
                const long start = idx;
                for (long k = 0; k < nodes_per_elem[e]; ++k) {
                    const long s = elem_nodes[e * max_nodes + k];
                    if (s == node) continue;
                    for (long cc = 0; cc < active_dofs[s]; ++cc, ++idx) col_inds[idx] = fmap[s] + cc;
                }
                cur[c] += idx - start;
            }
        }
        for (int cn = 0; cn < num_constraints; ++cn) {
            if (!con_contains(cn, di)) continue;
            for (long c = 0; c < nd; ++c) {
                long idx = rp[di + c] + cur[c];
                const long start = idx;
                for (long k = row_range[cn * 2]; k < row_range[cn * 2 + 1]; ++k, ++idx)
                    col_inds[idx] = num_system_dofs + k;
                cur[c] += idx - start;
            }
        }
    }
    // src/solver/compute_constraints_col_inds.hpp:51-59
    for (int c = 0; c < num_constraints; ++c) {
        for (long r = row_range[c * 2]; r < row_range[c * 2 + 1]; ++r) {
            long idx = rp[r + num_system_dofs];
            for (long k = 0; k < target_active[c]; ++k, ++idx) col_inds[idx] = target_table[c * 6 + k];
            for (long k = 0; k < base_active[c]; ++k, ++idx) col_inds[idx] = base_table[c * 6 + k];
        }
    }
    // KokkosSparse::sort_crs_graph (src/solver/create_full_matrix.hpp:62)
    if (sort_rows)
        for (int r = 0; r < num_dofs; ++r) std::sort(col_inds + rp[r], col_inds + rp[r + 1]);
    return nnz;
}

orc_model* orc_model_create(const kyn_model_desc* d, char* err, int errlen) {
    if (!d || d->num_nodes <= 0) {
        bad(err, errlen, "empty model");
        return nullptr;
    }
    auto* m = new orc_model();
    const int nn = d->num_nodes;
    m->num_nodes = nn;
    m->x0.assign(d->node_x0, d->node_x0 + nn * 7);
    m->q.resize(nn * 7);
    for (int n = 0; n < nn; ++n) {
        const double id[7] = {0., 0., 0., 1., 0., 0., 0.};
        for (int c = 0; c < 7; ++c) m->q[n * 7 + c] = d->node_u ? d->node_u[n * 7 + c] : id[c];
    }
    m->v.assign(nn * 6, 0.);
    m->vd.assign(nn * 6, 0.);
    if (d->node_v) m->v.assign(d->node_v, d->node_v + nn * 6);
    if (d->node_vd) m->vd.assign(d->node_vd, d->node_vd + nn * 6);
    // src/model/copy_nodes_to_state.hpp:14-60
    m->a = m->vd;
    m->f.assign(nn * 6, 0.);
    m->q_prev = m->q;
    m->q_delta.assign(nn * 6, 0.);
    m->x.assign(nn * 7, 0.);
    m->tangent.assign(nn * 36, 0.);
    update_global_position(*m);
    for (int c = 0; c < 3; ++c) m->gravity[c] = d->gravity[c];

    // src/elements/beams/create_beams.hpp:27-165
    m->beams.resize(d->num_beams);
    for (int e = 0; e < d->num_beams; ++e) {
        OBeam& B = m->beams[e];
        const int n0 = d->beam_node_offsets[e], n1 = d->beam_node_offsets[e + 1];
        const int s0 = d->beam_section_offsets[e], s1 = d->beam_section_offsets[e + 1];
        const int q0 = d->beam_qp_offsets[e], q1 = d->beam_qp_offsets[e + 1];
        B.N = n1 - n0;
        B.Q = q1 - q0;
        if (B.N < 2 || B.Q < 1 || s1 - s0 < 1) {
            bad(err, errlen, "beam needs >= 2 nodes, >= 1 qp, >= 1 section");
            delete m;
            return nullptr;
        }
        B.node_ids.assign(d->beam_node_ids + n0, d->beam_node_ids + n1);
        for (int id : B.node_ids) {
            if (id < 0 || id >= nn) {
                bad(err, errlen, "beam node id out of range");
                delete m;
                return nullptr;
            }
        }
        const int N = B.N, Q = B.Q;
        std::vector<double> node_xi(N);
        for (int n = 0; n < N; ++n) node_xi[n] = 2. * d->node_s[B.node_ids[n]] - 1.;
        B.phi.resize(N * Q);
        B.dphi.resize(N * Q);
        B.w.resize(Q);
        std::vector<double> wts;
        for (int qp = 0; qp < Q; ++qp) {
            const double xi = d->qp_xi[q0 + qp];
            B.w[qp] = d->qp_weight[q0 + qp];
            lagrange_interp(xi, node_xi, wts);
            for (int n = 0; n < N; ++n) B.phi[n * Q + qp] = wts[n];
            lagrange_deriv(xi, node_xi, wts);
            for (int n = 0; n < N; ++n) B.dphi[n * Q + qp] = wts[n];
        }
        // populate_element_views.hpp:90-141 (linear section interpolation)
        std::vector<double> sec_xi(s1 - s0);
        for (int s = s0; s < s1; ++s) sec_xi[s - s0] = 2. * d->section_position[s] - 1.;
        B.mstar.assign(Q * 36, 0.);
        B.cstar.assign(Q * 36, 0.);
        for (int qp = 0; qp < Q; ++qp) {
            linear_interp(d->qp_xi[q0 + qp], sec_xi, wts);
            for (int s = 0; s < s1 - s0; ++s) {
                for (int k = 0; k < 36; ++k) {
                    B.mstar[qp * 36 + k] += d->section_mass[(s0 + s) * 36 + k] * wts[s];
                    B.cstar[qp * 36 + k] += d->section_stiffness[(s0 + s) * 36 + k] * wts[s];
                }
            }
        }
        // interpolate_QP_rotation.hpp / interpolation_operations.hpp InterpQuaternion
        B.r0.resize(Q * 4);
        for (int qp = 0; qp < Q; ++qp) {
            double t[4] = {0., 0., 0., 0.};
            for (int n = 0; n < N; ++n) {
                const double phi = B.phi[n * Q + qp];
                for (int c = 0; c < 4; ++c) t[c] += m->x0[B.node_ids[n] * 7 + 3 + c] * phi;
            }
            const double len = std::sqrt(std::pow(t[0], 2) + std::pow(t[1], 2) +
                                         std::pow(t[2], 2) + std::pow(t[3], 2));
            if (len == 0.) {
                B.r0[qp * 4] = 1.;
                B.r0[qp * 4 + 1] = B.r0[qp * 4 + 2] = B.r0[qp * 4 + 3] = 0.;
            } else {
                for (int c = 0; c < 4; ++c) B.r0[qp * 4 + c] = t[c] / len;
            }
        }
        // calculate_jacobian.hpp:36-76
        std::vector<double> nx0(N * 7);
        for (int n = 0; n < N; ++n)
            for (int c = 0; c < 7; ++c) nx0[n * 7 + c] = m->x0[B.node_ids[n] * 7 + c];
        B.x0p.resize(Q * 3);
        B.jac.resize(Q);
        orc_calc_jacobian(N, Q, B.dphi.data(), nx0.data(), B.x0p.data(), B.jac.data());
        B.fx.assign(N * 6, 0.);
        B.fe.assign(Q * 6, 0.);
        B.residual.assign(N * 6, 0.);
        B.sysmat.assign(N * N * 36, 0.);
        B.eft.assign(N * 6, 0);
    }

    // src/elements/masses/create_masses.hpp, src/elements/springs/create_springs.hpp
    m->masses.resize(d->num_masses > 0 ? d->num_masses : 0);
    for (int e = 0; e < d->num_masses; ++e) {
        OMass& M = m->masses[e];
        M.node = d->mass_node[e];
        if (M.node < 0 || M.node >= nn) {
            bad(err, errlen, "mass node out of range");
            delete m;
            return nullptr;
        }
        for (int k = 0; k < 36; ++k) M.mstar[k] = d->mass_matrix[e * 36 + k];
        for (int c = 0; c < 4; ++c) M.r0[c] = m->x0[M.node * 7 + 3 + c];
    }
    m->springs.resize(d->num_springs > 0 ? d->num_springs : 0);
    for (int e = 0; e < d->num_springs; ++e) {
        OSpring& S = m->springs[e];
        S.n1 = d->spring_nodes[2 * e];
        S.n2 = d->spring_nodes[2 * e + 1];
        if (S.n1 < 0 || S.n1 >= nn || S.n2 < 0 || S.n2 >= nn || S.n1 == S.n2) {
            bad(err, errlen, "spring nodes out of range");
            delete m;
            return nullptr;
        }
        for (int c = 0; c < 3; ++c) S.x0[c] = m->x0[S.n2 * 7 + c] - m->x0[S.n1 * 7 + c];
        S.k = d->spring_stiffness[e];
        S.l_ref = d->spring_length[e];
    }

    // src/constraints/constraints.hpp:76-266
    m->cons.resize(d->num_constraints);
    long start_row = 0;
    for (int c = 0; c < d->num_constraints; ++c) {
        OConstraint& C = m->cons[c];
        C.type = d->constraint_type[c];
        const bool joint = C.type == KYN_CONSTRAINT_RIGID_JOINT || C.type == KYN_CONSTRAINT_ROTATION_CONTROL ||
                           C.type == KYN_CONSTRAINT_REVOLUTE_JOINT ||
                           C.type == KYN_CONSTRAINT_RIGID_JOINT_6DOF_TO_3DOF;
        const bool three = C.type >= KYN_CONSTRAINT_FIXED_BC_3DOF && C.type <= KYN_CONSTRAINT_RIGID_JOINT_6DOF_TO_3DOF;
        if (C.type != KYN_CONSTRAINT_FIXED_BC && C.type != KYN_CONSTRAINT_PRESCRIBED_BC && !joint && !three) {
            bad(err, errlen, "constraint type outside this path");
            delete m;
            return nullptr;
        }
        C.base = d->constraint_base_node ? d->constraint_base_node[c] : 0;
        C.target = d->constraint_target_node[c];
        if (C.target < 0 || C.target >= nn) {
            bad(err, errlen, "constraint node out of range");
            delete m;
            return nullptr;
        }
        if (joint && (C.base < 0 || C.base >= nn || C.base == C.target)) {
            bad(err, errlen, "joint base node out of range");
            delete m;
            return nullptr;
        }
        C.base_active = joint ? 6 : 0;
        C.target_active = three ? 3 : 6;
        // src/constraints/constraint_type.hpp NumRowsForConstraint: 5 for a revolute
        // joint, 3 for the three-row constraints on position-only nodes
        const int rows = C.type == KYN_CONSTRAINT_REVOLUTE_JOINT ? 5 : three ? 3 : 6;
        C.row_first = start_row;
        C.row_last = start_row + rows;
        start_row += rows;
        const double axis[3] = {d->constraint_axis ? d->constraint_axis[c * 3] : 0.,
                                d->constraint_axis ? d->constraint_axis[c * 3 + 1] : 0.,
                                d->constraint_axis ? d->constraint_axis[c * 3 + 2] : 0.};
        if (C.type == KYN_CONSTRAINT_FIXED_BC || C.type == KYN_CONSTRAINT_FIXED_BC_3DOF) {
            for (int k = 0; k < 3; ++k) C.X0[k] = m->x0[C.target * 7 + k] - axis[k];
        } else if (joint) {
            // src/constraints/constraints.hpp:268-290: relative position target - base
            for (int k = 0; k < 3; ++k) C.X0[k] = m->x0[C.target * 7 + k] - m->x0[C.base * 7 + k];
            if (C.type == KYN_CONSTRAINT_ROTATION_CONTROL) {
                // axes row 0 = UnitVector(axis) (src/constraints/constraints.hpp:321-328)
                const double nrm = std::sqrt(axis[0] * axis[0] + axis[1] * axis[1] + axis[2] * axis[2]);
                if (!(nrm > 0.)) {
                    bad(err, errlen, "rotation control needs a nonzero axis");
                    delete m;
                    return nullptr;
                }
                for (int k = 0; k < 3; ++k) C.axis[k] = axis[k] / nrm;
            }
            if (C.type == KYN_CONSTRAINT_REVOLUTE_JOINT) {
                // src/constraints/constraints.hpp:294-319: x_hat = unit(axis), or
                // unit(X0) for a zero axis; the frame is the rotation taking
                // (1, 0, 0) to x_hat, its rows the joint axes.
                const double na = std::sqrt(axis[0] * axis[0] + axis[1] * axis[1] + axis[2] * axis[2]);
                const double* src = na != 0. ? axis : C.X0;
                const double ns = std::sqrt(src[0] * src[0] + src[1] * src[1] + src[2] * src[2]);
                if (!(ns > 0.)) {
                    bad(err, errlen, "revolute joint needs an axis or distinct node positions");
                    delete m;
                    return nullptr;
                }
                const double xh[3] = {src[0] / ns, src[1] / ns, src[2] / ns};
                const double cp[3] = {0., -xh[2], xh[1]};  // (1, 0, 0) x x_hat
                const double dp = xh[0];
                if (!(1. + dp > 0.)) {
                    bad(err, errlen, "revolute joint axis along -x is outside this path");
                    delete m;
                    return nullptr;
                }
                const double k = 1. / (1. + dp);
                double* R = C.axes;
                R[0] = cp[0] * cp[0] * k + dp;
                R[1] = cp[1] * cp[0] * k + cp[2];
                R[2] = cp[2] * cp[0] * k - cp[1];
                R[3] = cp[0] * cp[1] * k - cp[2];
                R[4] = cp[1] * cp[1] * k + dp;
                R[5] = cp[2] * cp[1] * k + cp[0];
                R[6] = cp[0] * cp[2] * k + cp[1];
                R[7] = cp[1] * cp[2] * k - cp[0];
                R[8] = cp[2] * cp[2] * k + dp;
            }
        } else {
            const double idq[7] = {0., 0., 0., 1., 0., 0., 0.};
            for (int k = 0; k < 7; ++k)
                C.input[k] = d->constraint_initial_displacement
                                 ? d->constraint_initial_displacement[c * 7 + k]
                                 : idq[k];
        }
    }

    // src/dof_management/assemble_node_freedom_allocation_table.hpp
    m->sig.assign(nn, 0U);
    for (auto& B : m->beams)
        for (int id : B.node_ids) m->sig[id] |= 0b111111U;
    for (auto& M : m->masses) m->sig[M.node] |= 0b111111U;
    for (auto& S : m->springs) {  // JustPosition
        m->sig[S.n1] |= 0b111000U;
        m->sig[S.n2] |= 0b111000U;
    }
    for (auto& C : m->cons) {
        // FreedomSignature: JustPosition on the target of a three-row constraint
        m->sig[C.target] |= (C.target_active == 3) ? 0b111000U : 0b111111U;
        if (C.base_active) m->sig[C.base] |= 0b111111U;
    }
    m->active.resize(nn);
    for (int n = 0; n < nn; ++n) m->active[n] = count_bits(m->sig[n]);
    // compute_node_freedom_map_table.hpp
    m->fmap.assign(nn, 0);
    for (int n = 0; n + 1 < nn; ++n) m->fmap[n + 1] = m->fmap[n] + m->active[n];
    // create_element_freedom_table.hpp / create_constraint_freedom_table.hpp
    for (auto& B : m->beams)
        for (int n = 0; n < B.N; ++n)
            for (int c = 0; c < 6; ++c) B.eft[n * 6 + c] = m->fmap[B.node_ids[n]] + c;
    for (auto& M : m->masses)
        for (int c = 0; c < 6; ++c) M.eft[c] = m->fmap[M.node] + c;
    for (auto& S : m->springs)
        for (int c = 0; c < 3; ++c) {
            S.eft[0][c] = m->fmap[S.n1] + c;
            S.eft[1][c] = m->fmap[S.n2] + c;
        }
    for (auto& C : m->cons) {
        for (long c = 0; c < m->active[C.target]; ++c) C.target_table[c] = m->fmap[C.target] + c;
        for (int c = 0; c < 6; ++c) C.base_table[c] = C.base_active ? m->fmap[C.base] + c : 0;
    }
    m->nsys = 0;
    for (int n = 0; n < nn; ++n) m->nsys += m->active[n];
    m->ndofs = m->nsys + start_row;

    // src/solver/create_full_matrix.hpp:27-73
    // element connectivity in the order beams, masses, springs
    int maxn = 2;
    for (auto& B : m->beams) maxn = std::max(maxn, B.N);
    const size_t ne = m->beams.size() + m->masses.size() + m->springs.size();
    std::vector<long> npe(ne), en(ne * maxn, 0);
    size_t e_at = 0;
    for (size_t e = 0; e < m->beams.size(); ++e, ++e_at) {
        npe[e_at] = m->beams[e].N;
        for (int k = 0; k < m->beams[e].N; ++k) en[e_at * maxn + k] = m->beams[e].node_ids[k];
    }
    for (auto& M : m->masses) {
        npe[e_at] = 1;
        en[e_at * maxn] = M.node;
        ++e_at;
    }
    for (auto& S : m->springs) {
        npe[e_at] = 2;
        en[e_at * maxn] = S.n1;
        en[e_at * maxn + 1] = S.n2;
        ++e_at;
    }
    const int nc = static_cast<int>(m->cons.size());
    std::vector<long> ba(nc), ta(nc), bt(nc * 6), tt(nc * 6), rr(nc * 2);
    for (int c = 0; c < nc; ++c) {
        ba[c] = m->cons[c].base_active;
        ta[c] = m->cons[c].target_active;
        for (int k = 0; k < 6; ++k) {
            bt[c * 6 + k] = m->cons[c].base_table[k];
            tt[c * 6 + k] = m->cons[c].target_table[k];
        }
        rr[c * 2] = m->cons[c].row_first;
        rr[c * 2 + 1] = m->cons[c].row_last;
    }
    m->row_ptrs.resize(m->ndofs + 1);
    const long nnz = orc_crs_build(static_cast<int>(m->nsys), static_cast<int>(m->ndofs), nn,
                                   m->active.data(), m->fmap.data(),
                                   static_cast<int>(ne), maxn, npe.data(), en.data(),
                                   nc, ba.data(), ta.data(), bt.data(), tt.data(), rr.data(),
                                   m->row_ptrs.data(), nullptr, 1);
    m->col_inds.resize(nnz);
    orc_crs_build(static_cast<int>(m->nsys), static_cast<int>(m->ndofs), nn, m->active.data(),
                  m->fmap.data(), static_cast<int>(ne), maxn, npe.data(), en.data(),
                  nc, ba.data(), ta.data(), bt.data(), tt.data(), rr.data(), m->row_ptrs.data(),
                  m->col_inds.data(), 1);
    m->values.assign(nnz, 0.);
    m->b.assign(m->ndofs, 0.);
    m->xsol.assign(m->ndofs, 0.);
    return m;
}

void orc_model_destroy(orc_model* m) { delete m; }

void orc_set_solver_mode(orc_model* m, int mode) {
    if (m) m->solver_mode = mode;
}

int orc_model_info(const orc_model* m, kyn_model_info* info) {
    if (!m || !info) return KYN_ERR_INVALID;
    info->num_nodes = m->num_nodes;
    info->num_beams = static_cast<int32_t>(m->beams.size());
    info->num_constraints = static_cast<int32_t>(m->cons.size());
    info->num_system_dofs = static_cast<int32_t>(m->nsys);
    info->num_dofs = static_cast<int32_t>(m->ndofs);
    info->nnz = static_cast<int32_t>(m->col_inds.size());
    int mn = 0, mq = 0;
    for (auto& B : m->beams) {
        mn = std::max(mn, B.N);
        mq = std::max(mq, B.Q);
    }
    info->max_beam_nodes = mn;
    info->max_beam_qps = mq;
    info->device_bytes = 0;
    info->condensed_dofs = 0;
    return KYN_OK;
}

int orc_set_loads(orc_model* m, int which, const double* values) {
    if (!m || !values) return KYN_ERR_INVALID;
    if (which == KYN_LOAD_NODE_FX) {
        long k = 0;
        for (auto& B : m->beams)
            for (int n = 0; n < B.N; ++n)
                for (int c = 0; c < 6; ++c) B.fx[n * 6 + c] = values[k++ ];
        return KYN_OK;
    }
    if (which == KYN_LOAD_STATE_F) {
        std::copy(values, values + m->num_nodes * 6, m->f.begin());
        return KYN_OK;
    }
    return KYN_ERR_INVALID;
}

int orc_set_prescribed(orc_model* m, int cid, const double u[7]) {
    if (!m || cid < 0 || cid >= static_cast<int>(m->cons.size())) return KYN_ERR_INVALID;
    for (int k = 0; k < 7; ++k) m->cons[cid].input[k] = u[k];
    return KYN_OK;
}

int orc_step(orc_model* m, const kyn_step_params* p, int* iters) {
    if (!m || !p) return KYN_ERR_INVALID;
    return step_impl(*m, make_params(p), iters);
}

int orc_predict_and_assemble(orc_model* m, const kyn_step_params* p) {
    if (!m || !p) return KYN_ERR_INVALID;
    const Params P = make_params(p);
    predict(*m, P);
    for (auto& C : m->cons)
        for (int c = 0; c < 6; ++c) C.lambda[c] = C.sys_res[c] = 0.;
    assemble(*m, P);
    return KYN_OK;
}

int orc_get_state(const orc_model* m, int field, double* out) {
    if (!m || !out) return KYN_ERR_INVALID;
    const std::vector<double>* src = nullptr;
    switch (field) {
        case KYN_FIELD_X0: src = &m->x0; break;
        case KYN_FIELD_X: src = &m->x; break;
        case KYN_FIELD_Q: src = &m->q; break;
        case KYN_FIELD_Q_PREV: src = &m->q_prev; break;
        case KYN_FIELD_Q_DELTA: src = &m->q_delta; break;
        case KYN_FIELD_V: src = &m->v; break;
        case KYN_FIELD_VD: src = &m->vd; break;
        case KYN_FIELD_A: src = &m->a; break;
        case KYN_FIELD_F: src = &m->f; break;
        case KYN_FIELD_TANGENT: src = &m->tangent; break;
        case KYN_FIELD_LAMBDA: {
            for (size_t c = 0; c < m->cons.size(); ++c)
                for (int k = 0; k < 6; ++k) out[c * 6 + k] = m->cons[c].lambda[k];
            return KYN_OK;
        }
        case KYN_FIELD_CONSTRAINT_OUTPUT: {
            for (size_t c = 0; c < m->cons.size(); ++c)
                for (int k = 0; k < 3; ++k) out[c * 3 + k] = m->cons[c].output[k];
            return KYN_OK;
        }
        default: return KYN_ERR_INVALID;
    }
    std::copy(src->begin(), src->end(), out);
    return KYN_OK;
}

int orc_get_crs(const orc_model* m, int* rp, int* ci, double* vals) {
    if (!m) return KYN_ERR_INVALID;
    if (rp)
        for (size_t i = 0; i < m->row_ptrs.size(); ++i) rp[i] = static_cast<int>(m->row_ptrs[i]);
    if (ci)
        for (size_t i = 0; i < m->col_inds.size(); ++i) ci[i] = static_cast<int>(m->col_inds[i]);
    if (vals) std::copy(m->values.begin(), m->values.end(), vals);
    return KYN_OK;
}

int orc_get_system_vectors(const orc_model* m, double* rhs, double* sol) {
    if (!m) return KYN_ERR_INVALID;
    if (rhs) std::copy(m->b.begin(), m->b.end(), rhs);
    if (sol) std::copy(m->xsol.begin(), m->xsol.end(), sol);
    return KYN_OK;
}

int orc_get_convergence(const orc_model* m, double* errs, int* n) {
    if (!m) return KYN_ERR_INVALID;
    if (errs) std::copy(m->conv.begin(), m->conv.end(), errs);
    if (n) *n = static_cast<int>(m->conv.size());
    return KYN_OK;
}

int orc_get_element_terms(const orc_model* m, int e, double* residual, double* sysmat) {
    if (!m || e < 0 || e >= static_cast<int>(m->beams.size())) return KYN_ERR_INVALID;
    const OBeam& B = m->beams[e];
    if (residual) std::copy(B.residual.begin(), B.residual.end(), residual);
    if (sysmat) std::copy(B.sysmat.begin(), B.sysmat.end(), sysmat);
    return KYN_OK;
}

// FLOP tally of the counting build (0 in the normal one): reset, then read
// after a call to count the operations it made.
void orc_flops_reset() {
#ifdef ORC_COUNT_FLOPS
    g_flops = 0;
    g_qp_flops = 0;
#endif
}
long long orc_flops_read(int qp_only) {
#ifdef ORC_COUNT_FLOPS
    return qp_only ? g_qp_flops : g_flops;
#else
    (void)qp_only;
    return 0;
#endif
}

long orc_run_batch_record(orc_model** models, int n, const kyn_step_params* p, int first_step,
                          int steps, const double* amp, const double* freq, int nthreads,
                          double* seconds, int* status, int* iters_out) {
    const Params P = make_params(p);
    long converged = 0;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
    const auto t0 = std::chrono::steady_clock::now();
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : converged)
    for (int i = 0; i < n; ++i) {
        orc_model& m = *models[i];
        for (int k = 0; k < steps; ++k) {
            if (amp && freq && !m.beams.empty()) {
                OBeam& B = m.beams[0];
                const double t = P.h * static_cast<double>(first_step + k + 1);
                B.fx[(B.N - 1) * 6 + 2] = amp[i] * std::sin(2. * M_PI * freq[i] * t);
            }
            int it = 0;
            int st = step_impl(m, P, &it);
            // The reference's Newton loop runs while err > 1, so a NaN error
            // ends it and Step() returns true (src/step/step.hpp:54); the state
            // evolves exactly as there, but for counting converged beam-steps a
            // step whose last error is not finite is reported non-finite, as
            // the GPU path reports it.
            if (st == KYN_OK && !m.conv.empty() && !std::isfinite(m.conv.back())) st = KYN_ERR_NONFINITE;
            if (status) status[static_cast<long>(i) * steps + k] = st;
            if (iters_out) iters_out[static_cast<long>(i) * steps + k] = it;
            if (st == KYN_OK) ++converged;
        }
    }
    const auto t1 = std::chrono::steady_clock::now();
    if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
    return converged;
}

long orc_run_batch(orc_model** models, int n, const kyn_step_params* p, int steps,
                   const double* amp, const double* freq, int nthreads, double* seconds,
                   int* iters_total) {
    std::vector<int> it(static_cast<size_t>(n) * (steps > 0 ? steps : 0), 0);
    const long conv = orc_run_batch_record(models, n, p, 0, steps, amp, freq, nthreads, seconds,
                                           nullptr, it.data());
    long total = 0;
    for (int v : it) total += v;
    if (iters_total) *iters_total = static_cast<int>(total);
    return conv;
}

// ---- kernel-level entry points --------------------------------------------

void orc_lagrange_interp_weights(double x, const double* xs, int n, double* w) {
    std::vector<double> v(xs, xs + n), out;
    lagrange_interp(x, v, out);
    std::copy(out.begin(), out.end(), w);
}

void orc_lagrange_deriv_weights(double x, const double* xs, int n, double* w) {
    std::vector<double> v(xs, xs + n), out;
    lagrange_deriv(x, v, out);
    std::copy(out.begin(), out.end(), w);
}

// src/math/interpolation.hpp GenerateGLLPoints
void orc_gll_points(int order, double* pts) {
    const int nn = order + 1;
    std::vector<double> g(nn, 0.);
    g.front() = -1.;
    g.back() = 1.;
    auto legendre = [](int n, double x) {
        if (n == 0) return 1.;
        if (n == 1) return x;
        double p2 = 1., p1 = x, p = 0.;
        for (int i = 2; i <= n; ++i) {
            const double id = static_cast<double>(i);
            p = ((2. * id - 1.) * x * p1 - (id - 1.) * p2) / id;
            p2 = p1;
            p1 = p;
        }
        return p;
    };
    for (int i = 1; i < order; ++i) {
        double x = -std::cos(static_cast<double>(i) * M_PI / static_cast<double>(order));
        for (int it = 0; it < 1000; ++it) {
            const double xo = x;
            const double pn = legendre(nn - 1, x), pm = legendre(nn - 2, x);
            const double num = x * pn - pm;
            const double den = static_cast<double>(nn) * pn;
            x -= num / den;
            if (std::abs(x - xo) <= std::numeric_limits<double>::epsilon()) break;
        }
        g[i] = x;
    }
    std::copy(g.begin(), g.end(), pts);
}

void orc_rotate_section(const double xr[4], const double cstar[36], double out[36]) {
    rotate_section(xr, cstar, out);
}

void orc_calc_strain(const double x0p[3], const double up[3], const double r[4],
                     const double rp[4], double strain[6]) {
    calc_strain(x0p, up, r, rp, strain);
}

void orc_calc_fc(const double cuu[36], const double strain[6], double fc[6]) {
    gemv(false, 6, 6, 1., cuu, 6, strain, 0., fc);
}

void orc_calc_fd(const double ss[9], const double fc[6], double fd[6]) {
    for (int i = 0; i < 6; ++i) fd[i] = 0.;
    gemv(true, 3, 3, 1., ss, 3, fc, 0., fd + 3);
}

void orc_calc_ouu(const double cuu[36], const double ss[9], const double mt[9],
                  const double nt[9], double out[36]) {
    calc_ouu(cuu, ss, mt, nt, out);
}

void orc_calc_puu(const double cuu[36], const double ss[9], const double nt[9], double out[36]) {
    calc_puu(cuu, ss, nt, out);
}

void orc_calc_quu(const double cuu[36], const double ss[9], const double nt[9], double out[36]) {
    calc_quu(cuu, ss, nt, out);
}

// src/elements/beams/calculate_jacobian.hpp:36-76
void orc_calc_jacobian(int nn, int nq, const double* sd, const double* nx0, double* x0p,
                       double* jac) {
    for (int qp = 0; qp < nq; ++qp) {
        double t[3] = {0., 0., 0.};
        for (int n = 0; n < nn; ++n) {
            const double phi = sd[n * nq + qp];
            for (int c = 0; c < 3; ++c) t[c] += nx0[n * 7 + c] * phi;
        }
        for (int c = 0; c < 3; ++c) x0p[qp * 3 + c] = t[c];
    }
    for (int qp = 0; qp < nq; ++qp) {
        const double j = std::sqrt(std::pow(x0p[qp * 3], 2.) + std::pow(x0p[qp * 3 + 1], 2.) +
                                   std::pow(x0p[qp * 3 + 2], 2.));
        jac[qp] = j;
        for (int c = 0; c < 3; ++c) x0p[qp * 3 + c] /= j;
    }
}

// src/system/beams/integrate_residual_vector.hpp:33-50
void orc_integrate_residual(int nn, int nq, const double* w, const double* jac,
                            const double* phi, const double* dphi, const double* fx,
                            const double* fc, const double* fd, const double* fi,
                            const double* fe, const double* fg, double* out) {
    for (int n = 0; n < nn; ++n) {
        double loc[6] = {0, 0, 0, 0, 0, 0};
        for (int qp = 0; qp < nq; ++qp) {
            const double weight = w[qp];
            const double cc = weight * dphi[n * nq + qp];
            const double cd = weight * jac[qp] * phi[n * nq + qp];
            for (int c = 0; c < 6; ++c)
                loc[c] += cc * fc[qp * 6 + c] +
                          cd * (fd[qp * 6 + c] + fi[qp * 6 + c] - fe[qp * 6 + c] - fg[qp * 6 + c]);
        }
        for (int c = 0; c < 6; ++c) out[n * 6 + c] = loc[c] - fx[n * 6 + c];
    }
}

// src/system/beams/integrate_stiffness_matrix.hpp:35-96
void orc_integrate_stiffness(int nn, int nq, const double* w, const double* jac,
                             const double* phi, const double* dphi, const double* kuu,
                             const double* puu, const double* cuu, const double* ouu,
                             const double* quu, double* out) {
    for (int i = 0; i < nn; ++i) {
        for (int j = 0; j < nn; ++j) {
            double loc[36] = {};
            for (int qp = 0; qp < nq; ++qp) {
                const double ww = w[qp], J = jac[qp];
                const double p1 = phi[i * nq + qp], p2 = phi[j * nq + qp];
                const double d1 = dphi[i * nq + qp], d2 = dphi[j * nq + qp];
                const double K = (p1 * p2) * (ww * J);
                const double P = (p1 * d2) * ww;
                const double C = (d1 * d2) * (ww / J);
                const double O = (d1 * p2) * ww;
                for (int c = 0; c < 36; ++c)
                    loc[c] = loc[c] + K * (kuu[qp * 36 + c] + quu[qp * 36 + c]) +
                             P * puu[qp * 36 + c] + C * cuu[qp * 36 + c] + O * ouu[qp * 36 + c];
            }
            for (int c = 0; c < 36; ++c) out[(i * nn + j) * 36 + c] = loc[c];
        }
    }
}

// src/system/beams/integrate_inertia_matrix.hpp:32-78
void orc_integrate_inertia(int nn, int nq, const double* w, const double* jac,
                           const double* phi, const double* muu, const double* guu,
                           double bp, double gp, double* out) {
    for (int i = 0; i < nn; ++i) {
        for (int j = 0; j < nn; ++j) {
            double loc[36] = {};
            for (int qp = 0; qp < nq; ++qp) {
                const double coeff = phi[i * nq + qp] * phi[j * nq + qp] * w[qp] * jac[qp];
                for (int c = 0; c < 36; ++c) {
                    const double contribution = bp * muu[qp * 36 + c] + gp * guu[qp * 36 + c];
                    loc[c] = loc[c] + coeff * contribution;
                }
            }
            for (int c = 0; c < 36; ++c) out[(i * nn + j) * 36 + c] = loc[c];
        }
    }
}

void orc_inertial_qp(double, const double mstar[36], const double r0[4], const double r[4],
                     const double uddot[3], const double omega[3], const double omegadot[3],
                     const double gravity[3], double fi[6], double fg[6], double muu[36],
                     double guu[36], double kuu[36]) {
    inertial_qp(mstar, r0, r, uddot, omega, omegadot, gravity, fi, fg, muu, guu, kuu);
}

void orc_tangent_operator(double h, const double qdelta[6], double t_stored[36]) {
    tangent_operator(h, qdelta, t_stored);
}

// Kernel-level forms of the revolute joint's residual and gradients, torque
// and output (the oracle's update_revolute_joint / revolute_output on a
// two-node model: base node 0, target node 1, identity tangents), for the
// reference's unit tests test_calculate_revolute_joint_{constraint,force,output}.cpp.
void orc_revolute_joint(const double X0[3], const double axes[9], const double base_u[7],
                        const double target_u[7], double torque, double res[6], double base_grad[36],
                        double target_grad[36], double sys_res[6]) {
    orc_model m;
    m.num_nodes = 2;
    m.q.assign(base_u, base_u + 7);
    m.q.insert(m.q.end(), target_u, target_u + 7);
    m.tangent.assign(72, 0.);
    for (int n = 0; n < 2; ++n)
        for (int c = 0; c < 6; ++c) m.tangent[n * 36 + c * 7] = 1.;
    OConstraint C;
    C.type = KYN_CONSTRAINT_REVOLUTE_JOINT;
    C.base = 0;
    C.target = 1;
    for (int k = 0; k < 3; ++k) C.X0[k] = X0[k];
    for (int k = 0; k < 9; ++k) C.axes[k] = axes[k];
    C.input[0] = torque;
    update_revolute_joint(m, C);
    for (int k = 0; k < 6; ++k) {
        res[k] = C.res[k];
        sys_res[k] = C.sys_res[k];
    }
    for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j) {
            base_grad[i * 6 + j] = C.b_grad_trans[j * 6 + i];
            target_grad[i * 6 + j] = C.t_grad_trans[j * 6 + i];
        }
}

// Kernel-level form of the six-row constraints (FixedBC, PrescribedBC,
// RigidJoint, RotationControl with its raw axis) on a two-node model (base 0,
// target 1, identity tangents): residual and gradients, for the reference's
// unit tests test_calculate_{fixed_bc,prescribed_bc,rigid_joint,rotation_control}_constraint.cpp.
void orc_constraint_kernel(int type, const double X0[3], const double axis[3], const double input[7],
                           const double base_u[7], const double target_u[7], double res[6],
                           double base_grad[36], double target_grad[36]) {
    orc_model m;
    m.num_nodes = 2;
    m.q.assign(base_u, base_u + 7);
    m.q.insert(m.q.end(), target_u, target_u + 7);
    m.tangent.assign(72, 0.);
    for (int n = 0; n < 2; ++n)
        for (int c = 0; c < 6; ++c) m.tangent[n * 36 + c * 7] = 1.;
    OConstraint C;
    C.type = type;
    C.base = 0;
    C.target = 1;
    for (int k = 0; k < 3; ++k) {
        C.X0[k] = X0[k];
        C.axis[k] = axis[k];
    }
    for (int k = 0; k < 7; ++k) C.input[k] = input[k];
    update_constraint(m, C);
    for (int k = 0; k < 6; ++k) res[k] = C.res[k];
    for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j) {
            base_grad[i * 6 + j] = C.b_grad_trans[j * 6 + i];
            target_grad[i * 6 + j] = C.t_grad_trans[j * 6 + i];
        }
}

void orc_revolute_output(const double axes[9], const double u[7], const double udot[6],
                         const double uddot[6], double out[3]) {
    orc_model m;
    m.num_nodes = 1;
    m.q.assign(u, u + 7);
    m.v.assign(udot, udot + 6);
    m.vd.assign(uddot, uddot + 6);
    OConstraint C;
    C.type = KYN_CONSTRAINT_REVOLUTE_JOINT;
    C.target = 0;
    for (int k = 0; k < 9; ++k) C.axes[k] = axes[k];
    revolute_output(m, C);
    for (int k = 0; k < 3; ++k) out[k] = C.output[k];
}

}  // extern "C"
