// kyn_step_kernel.cuh -- fused per-beam time-step kernel for sm_100a.
//
// One CTA owns one beam element for a whole time step: predictor, every
// Newton iteration (tangent operator, quadrature-point physics, node-pair
// integration, assembly of the bordered constraint system, linear solve,
// convergence test, update) and the post-step update.  The beam system lives
// in shared memory for the whole step; HBM is touched only to read the beam's
// constant data and to read/write its resident state.  The beams of one model
// form a thread-block cluster and sum the model's convergence error through
// distributed shared memory, so every beam of a model takes the same Newton
// iterations as the reference's model-wide loop (src/step/step.hpp:54-83).
// Models without beam elements whose constraints are more than single-node
// BCs run in dense_kernel (the bordered system with a pivoted LU).
//
// Linear solve: the reference factors the whole bordered system with a
// sparse direct solver (src/step/solve_system.hpp:27-31).  Here the
// single-node boundary conditions are eliminated exactly: their gradient
// B = grad*T and transpose grad^T are block-diagonal with an identity
// translational block (src/constraints/calculate_fixed_bc_constraint.hpp,
// calculate_prescribed_bc_constraint.hpp), so the constrained node's
// correction follows from a 3x3 solve, the free-node block is factored by LU
// in shared memory, and the multipliers follow from the constrained rows.
#pragma once

#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include "../../include/kynema_b200.h"
#include "kyn_types.h"

namespace kyn {

namespace cg = cooperative_groups;

// ---- small math (src/math/quaternion_operations.hpp, vector_operations.hpp) --
__device__ __forceinline__ void quat_compose(const double* a, const double* b, double* o) {
    o[0] = a[0] * b[0] - a[1] * b[1] - a[2] * b[2] - a[3] * b[3];
    o[1] = a[0] * b[1] + a[1] * b[0] + a[2] * b[3] - a[3] * b[2];
    o[2] = a[0] * b[2] - a[1] * b[3] + a[2] * b[0] + a[3] * b[1];
    o[3] = a[0] * b[3] + a[1] * b[2] - a[2] * b[1] + a[3] * b[0];
}

// Entry (i,j) of the rotation matrix of unit quaternion q.
__host__ __device__ __forceinline__ double rot_entry(const double* q, int i, int j) {
    const double w = q[0], x = q[1], y = q[2], z = q[3];
    switch (i * 3 + j) {
        case 0: return w * w + x * x - y * y - z * z;
        case 1: return 2. * (x * y - w * z);
        case 2: return 2. * (x * z + w * y);
        case 3: return 2. * (x * y + w * z);
        case 4: return w * w - x * x + y * y - z * z;
        case 5: return 2. * (y * z - w * x);
        case 6: return 2. * (x * z - w * y);
        case 7: return 2. * (y * z + w * x);
        default: return w * w - x * x - y * y + z * z;
    }
}

// Entry (i,j) of tilde(v) (VecTilde).
__device__ __forceinline__ double tilde_e(const double* v, int i, int j) {
    if (i == j) return 0.;
    const int k = 3 - i - j;
    const double s = ((i + 1) % 3 == j) ? -1. : 1.;
    return s * v[k];
}

__device__ __forceinline__ void cross3(const double* a, const double* b, double* c) {
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
}

// Exponential map: rotation vector -> quaternion (RotationVectorToQuaternion,
// device form with factor 0 below 1e-12).
__device__ __forceinline__ void rotvec_to_quat(const double* phi, double* q) {
    const double angle = sqrt(phi[0] * phi[0] + phi[1] * phi[1] + phi[2] * phi[2]);
    double s, c;
    sincos(angle / 2., &s, &c);
    const double f = (fabs(angle) < 1.e-12) ? 0. : s / angle;
    q[0] = c;
    q[1] = phi[0] * f;
    q[2] = phi[1] * f;
    q[3] = phi[2] * f;
}

// Solve the 3x3 system M y = r (row-major M) by Cramer's rule; the matrices
// solved here (rotational blocks of the boundary-condition gradient) are
// close to rotations, so the determinant is far from zero.
__device__ inline bool solve3(const double* M, const double* r, double* y) {
    const double c00 = M[4] * M[8] - M[5] * M[7];
    const double c01 = M[5] * M[6] - M[3] * M[8];
    const double c02 = M[3] * M[7] - M[4] * M[6];
    const double det = M[0] * c00 + M[1] * c01 + M[2] * c02;
    if (!(fabs(det) > 0.)) return false;
    const double id = 1. / det;
    y[0] = (r[0] * c00 + M[1] * (M[5] * r[2] - r[1] * M[8]) + M[2] * (r[1] * M[7] - M[4] * r[2])) * id;
    y[1] = (M[0] * (r[1] * M[8] - M[5] * r[2]) + r[0] * c01 + M[2] * (M[3] * r[2] - r[1] * M[6])) * id;
    y[2] = (M[0] * (M[4] * r[2] - r[1] * M[7]) + M[1] * (r[1] * M[6] - M[3] * r[2]) + r[0] * c02) * id;
    return true;
}

// FP64 tensor-core product D += A B for one 8x8x4 tile (mma.sync m8n8k4 .f64).
// Fragment layout per lane l: a = A[l/4][l%4], b = B[l%4][l/4],
// d0/d1 = D[l/4][2(l%4)] / D[l/4][2(l%4)+1].
__device__ __forceinline__ void dmma884(double& d0, double& d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// ---- bulk copies into shared memory (cp.async.bulk, completion on an mbarrier) --
// One thread arms the barrier with the byte count and issues the copy; every
// thread that reads the data waits on the barrier's phase parity.  The copy
// is a plain (non-multicast) global -> own-CTA shared-memory transfer.
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
// src, dst 16-byte aligned, bytes a multiple of 16.  Every thread that
// accessed the destination through ordinary loads and stores runs
// proxy_fence_async_smem() before the CTA barrier that precedes this call.
__device__ __forceinline__ void proxy_fence_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
// Waits for phase `parity` of the barrier, at most kBulkWaitTries polls;
// false when it gave up.
constexpr int kBulkWaitTries = 1 << 22;
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    const uint32_t b = smem_u32(bar);
    for (int i = 0; i < kBulkWaitTries; ++i) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(b), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// Doubles of one beam system's per-point section data as it lies in the slab
// from x0' on: x0' [Q][3] (padded to even), r0 [Q][4], M* [Q][36], C* [Q][36]
// (SlabLayout keeps them contiguous); staged per Newton iteration.
__host__ __device__ inline int sec_doubles(int Q) { return ((3 * Q + 1) & ~1) + 76 * Q; }

// ---- shared-memory plan of one CTA --------------------------------------------
// The kernel runs with NT = 128, 256 or 512 threads (up to four, two or one
// CTAs per SM within the 128-register budget); NT/16 quadrature points are
// processed per pass and NT/32 warps share the GEMM-shaped phases.  More
// resident CTAs overlap more beams' serial sections (LU pivots); more warps
// per CTA shorten the parallel phases of one beam.
constexpr int kGroupScratch = 256;      // doubles of per-group scratch for QP math
constexpr int kPanel = 8;               // LU panel width
constexpr int kConStride = 96;          // doubles per constraint record in smem
constexpr int kHubSmem = 208;           // doubles of the hub record (hubsm)
constexpr int kDriveSmem = 600;         // doubles of the hub record of a drive train

// Per-group scratch (doubles) of the quadrature phase.
namespace grec {
constexpr int interp = 0;   // [20] interpolated sums
constexpr int rn = 20;      // [4] normalised r
constexpr int Rx = 24;      // [9] R(r o r0)
constexpr int Rr = 33;      // [9] R(r)
constexpr int st = 42;      // [6] strain
constexpr int Mu = 48;      // [36] Muu
constexpr int ms = 84;      // mass, eta[3], s = x0'+u' [3] at 88..90
constexpr int O12 = 92;     // [9]
constexpr int Gu = 101;     // [18]
constexpr int Kk = 119;     // [9]
constexpr int fcv = 128;    // [6]
constexpr int Cu = 136;     // [36] Cuu (rotated stiffness)
constexpr int mstar = 172;  // [36] sectional mass (material frame), staged from HBM
constexpr int cstar = 208;  // [36] sectional stiffness
constexpr int r0 = 244;     // [4]
constexpr int x0p = 248;    // [3]
}  // namespace grec

struct Smem {
    int A;              // TR [n6][ldA]; aliased by the per-group QP scratch
    int G;              // double [4Q][56] weighted quadrature blocks (integration GEMM)
    int Fc, Fdig;       // double [Q][6]
    int phi, dphi;      // double [Q][N]
    int dphiJ;          // double [Q][N]
    int qpw;            // double [Q][4]
    int q, q_prev, v, vd, a, qd;  // node state
    int T;              // double [N][9]
    int resid;          // double [N][6]
    int b;              // double [n6]  permuted rhs
    int xs;             // double [n6]  permuted solution
    int rpiv;           // double [n6]  reciprocal pivots
    int stage;          // double [64]  U12 tile staged by warp 0 during the LU
    int con;            // double [nc][kConStride]
    int red;            // double [2][NT/32 + 8]  (offset 0: cluster exchange)
    int hub;            // double [kHubSmem or kDriveSmem] hub state and records, or -1
    int pos;            // int [N]
    int sec;            // double [sec_doubles(Q)] staged sections, inside A's region after
                        // the group scratch (quadrature phase only)
    int bar;            // uint64 mbarrier of the section copies
    int bytes;
    int ldA;
};

// Entries of one slot of the Gauss-Jordan pivot buffers for (storage bytes,
// threads): 2 (RT * NT/16 + CT * 16) with the tile sizes GJTile below (the
// pivot pair's column and row entries).
__host__ __device__ constexpr int gj_slot_entries(int real_bytes, int nt) {
    return 2 * (real_bytes == 8 ? (nt == 128 ? 7 * 8 + 4 * 16 : nt == 256 ? 6 * 16 + 6 * 16 : 4 * 32 + 8 * 16)
                                : (nt == 128 ? 8 * 8 + 5 * 16 : nt == 256 ? 8 * 16 + 8 * 16 : 4 * 32 + 8 * 16));
}

// Bytes of the solve-phase scratch that lives in the G region (dead after the
// integration): the two pivot-buffer slots, then FP64 vectors of n6 entries
// (residual, second right-hand side, its solution, correction) and 4 * 16
// doubles of reductions.
__host__ __device__ inline int gj_vec_offset(int real_bytes, int nt) {
    return (2 * gj_slot_entries(real_bytes, nt) * real_bytes + 15) & ~15;
}
__host__ __device__ inline int gj_scratch_bytes(int N, int real_bytes, int nt) {
    return gj_vec_offset(real_bytes, nt) + 4 * 6 * N * 8 + 64 * 8;
}

// The system matrix and the quadrature scratch never live at the same time:
// A is assembled after the quadrature phase and consumed by the solve, so the
// two share one region; so do the sections staged for the next quadrature
// phase, copied in once the solve has read A for the last time.
// hub: 0 none, 1 a hub node, 2 a drive train (hub chain of 2 or 3 nodes).
__host__ __device__ inline Smem make_smem(int N, int Q, int nc, int real_bytes, int nt, int hub = 0) {
    Smem S{};
    int o = 0;
    auto take = [&](int bytes) {
        const int r = o;
        o += (bytes + 15) & ~15;
        return r;
    };
    const int n6 = 6 * N;
    S.ldA = n6 + 1;
    // The cluster exchange areas come first, so that every CTA of a model's
    // cluster finds them at the same offset whatever its beam's size.
    S.red = take(2 * (nt / 32 + 8) * 8);
    S.hub = hub ? take((hub > 1 ? kDriveSmem : kHubSmem) * 8) : -1;
    {
        const int a_bytes = n6 * S.ldA * real_bytes;
        const int g_bytes = (nt / 16) * kGroupScratch * 8;
        const int q_bytes = g_bytes + sec_doubles(Q) * 8;
        S.A = take(a_bytes > q_bytes ? a_bytes : q_bytes);
        S.sec = S.A + g_bytes;
    }
    // FP64 form: G in FP64, one k-step per point.  FP32 form: G in FP32 and
    // k-steps of two points (m16n8k8), so an odd Q gets one zero pad point.
    {
        const int g_bytes = 4 * (real_bytes == 4 ? (Q + 1) & ~1 : Q) * 56 * real_bytes;
        const int s_bytes = gj_scratch_bytes(N, real_bytes, nt);
        S.G = take(g_bytes > s_bytes ? g_bytes : s_bytes);
    }
    S.Fc = take(Q * 6 * 8);
    S.Fdig = take(Q * 6 * 8);
    S.phi = take(Q * N * 8);
    S.dphi = take(Q * N * 8);
    S.dphiJ = take(Q * N * 8);
    S.qpw = take(Q * 4 * 8);
    S.q = take(N * 7 * 8);
    S.q_prev = take(N * 7 * 8);
    S.v = take(N * 6 * 8);
    S.vd = take(N * 6 * 8);
    S.a = take(N * 6 * 8);
    S.qd = take(N * 6 * 8);
    S.T = take(N * 9 * 8);
    S.resid = take(N * 6 * 8);
    S.b = take(n6 * 8);
    S.xs = take(n6 * 8);
    S.rpiv = take(n6 * 8);
    S.stage = take(64 * 8);
    S.con = take((nc > 0 ? nc : 1) * kConStride * 8);
    S.pos = take(N * 4);
    S.bar = take(8);
    S.bytes = o;
    return S;
}

// Column layout of the integration GEMM's B operand G (56 columns).  The 54
// quantities of a node pair are L[r][c] (left 6x3 block, logical r*3+c),
// RS[r][k] (right block before the tangent, 18 + r*3+k) and RI[r][c] (right
// inertia block, 36 + r*3+c).  m8n8k4 leaves column 8*nt + 2*s + e of a tile
// row in lane s = lane%4, slot 2*nt + e; the layout puts the six values of
// two right-block rows (RS and RI) in one lane, so SM_ij = C_RS T_j + C_RI is
// formed from registers: lanes 0..2 own rows {2s, 2s+1} in slots 0..11 and two
// L values in slots 12..13 (lane 2: padding), lane 3 owns L[0..13].
__host__ __device__ inline int gcol_slot(int s, int t) { return 8 * (t >> 1) + 2 * s + (t & 1); }
__host__ __device__ inline int gcol(int logical) {
    if (logical < 18) {
        if (logical < 14) return gcol_slot(3, logical);
        if (logical < 16) return gcol_slot(0, 12 + logical - 14);
        return gcol_slot(1, 12 + logical - 16);
    }
    const bool ri = logical >= 36;
    const int e = logical - (ri ? 36 : 18);
    const int r = e / 3, k = e % 3;
    return gcol_slot(r >> 1, (r & 1) * 6 + (ri ? 3 : 0) + k);
}

// Constraint record layout inside Smem::con (doubles).
namespace conrec {
constexpr int Phi = 0;     // [6] residual
constexpr int Brot = 6;    // [9] rotational block of B = grad*T (row-major)
constexpr int AX = 15;     // [9] rotational block of grad^T  (= AX(C))
constexpr int Gl = 24;     // [6] grad^T lambda
constexpr int xl = 30;     // [6] multiplier correction
constexpr int lam = 36;    // [6] lambda
constexpr int inp = 42;    // [7] prescribed input
constexpr int yr = 49;     // [6] constrained-row residual b_r - A_r x
constexpr int R1X0 = 55;   // [3] rigid joint: R(hub) X0
constexpr int Btr = 58;    // [9] rigid joint: base block tilde(R1 X0) T_hub
constexpr int Brr = 67;    // [9] rigid joint: base block -AX(C) T_hub
constexpr int dr = 76;     // [6] drive train: root correction per unit shaft rotation
constexpr int wr = 82;     // [6] drive train: root test vector (G w = 0)
constexpr int s2 = 88;     // [6] drive train: A_r x2 of the second right-hand side
}  // namespace conrec

// Shared-memory record of a model's hub (doubles): the hub state in the slab
// layout (hubrec), the hub BC's constraint record, the hub correction, the
// hub multiplier correction, and the per-beam contributions exchanged over
// the cluster (double-buffered by iteration parity).
namespace hubsm {
constexpr int bc = 88;     // [kConStride] constraint record of the hub BC
constexpr int xh = 184;    // [6] hub correction
constexpr int xlh = 190;   // [6] hub multiplier correction (unconditioned)
constexpr int pub = 196;   // [2][6] sum over this beam's joints of G_base^T (lambda + x_lambda)
// drive train (records 1 and 2 of the hub chain, the revolute and rigid joints
// between them, and the vectors of the shaft-rotation elimination)
constexpr int n1 = 208;    // [kHubDoubles] chain record 1 (azimuth node)
constexpr int n2 = 296;    // [kHubDoubles] chain record 2 (hub node), if any
constexpr int rev = 384;   // [64] revolute joint record (revrec)
constexpr int ah = 448;    // [kConStride] rigid joint record 1 -> 2
constexpr int cA = 544;    // [6] record-1 correction at zero shaft rotation
constexpr int nA = 550;    // [6] record-1 correction per unit shaft rotation
constexpr int cH = 556;    // [6] record-2 correction at zero shaft rotation
constexpr int dH = 562;    // [6] record-2 correction per unit shaft rotation
constexpr int wA = 568;    // [6] record-1 test vector
constexpr int wH = 574;    // [6] record-2 test vector
constexpr int theta = 580; // shaft rotation of the Newton correction
constexpr int xt = 584;    // [2][8] this beam's part of the shaft equation (num, den,
                           // G_base^T lambda of its joints), exchanged over the cluster
}  // namespace hubsm

// Revolute joint record (doubles, at hubsm::rev).
namespace revrec {
constexpr int Phi = 0;     // [5] residual
constexpr int x = 5;       // [3] R(base) x0: joint axis
constexpr int y = 8;       // [3] R(target) y0
constexpr int z = 11;      // [3] R(target) z0
constexpr int xcz = 14;    // [3] x cross z
constexpr int xcy = 17;    // [3] x cross y
constexpr int Bt = 20;     // [2][3] rotational rows of G_target T_target
constexpr int Bb = 26;     // [2][3] rotational rows of G_base T_base
constexpr int sys = 32;    // [3] torque about R(target) x0
constexpr int lam = 35;    // [6] multipliers (5 used)
constexpr int xl = 41;     // [6] multiplier correction (unconditioned)
constexpr int GtL = 47;    // [6] G_target^T lambda
constexpr int GbL = 53;    // [6] G_base^T lambda
}  // namespace revrec

// TF32 tensor-core product D += A B for one 16x8x8 tile (mma.sync m16n8k8).
// Fragment layout per lane l (g = l/4, t = l%4): a = {A[g][t], A[g+8][t],
// A[g][t+4], A[g+8][t+4]}, b = {B[t][g], B[t+4][g]}, d = {D[g][2t], D[g][2t+1],
// D[g+8][2t], D[g+8][2t+1]}.
__device__ __forceinline__ void mma_tf32(float* d, const unsigned* a, const unsigned* b) {
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
        "{%8,%9}, {%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// x = hi + lo with hi, lo representable in TF32 (round to nearest, ties away).
__device__ __forceinline__ void split_tf32(float x, unsigned& hi, unsigned& lo) {
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(hi) : "f"(x));
    const float r = x - __uint_as_float(hi);
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(lo) : "f"(r));
}

// Writes SM_ij = [C_L | C_RS T_j + C_RI] of node pair (i, j), scaled by the
// conditioner, into the system matrix from one lane's integration-GEMM slots
// (column layout: gcol; slot(t) returns the lane's slot t).
template <typename TR, typename Slot>
__device__ __forceinline__ void store_pair_block(TR* A, int ldA, const int* pos, const double* sT,
                                                 int i, int jn, int s4, double cond, Slot slot) {
    TR* Arow = A + (6 * pos[i]) * ldA + 6 * pos[jn];
    if (s4 < 3) {
        const double* Tj = sT + jn * 9;
#pragma unroll
        for (int rr = 0; rr < 2; ++rr) {
            const int r = 2 * s4 + rr;
            // slots 6rr..6rr+2: RS[r][0..2]; 6rr+3..6rr+5: RI[r][0..2]
            double rs[3], ri[3];
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                rs[k] = slot(6 * rr + k);
                ri[k] = slot(6 * rr + 3 + k);
            }
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                double val = ri[c];
#pragma unroll
                for (int k = 0; k < 3; ++k) val += rs[k] * Tj[k * 3 + c];
                Arow[r * ldA + 3 + c] = static_cast<TR>(val * cond);
            }
        }
        if (s4 < 2) {
            // slots 12, 13: L[14 + 2 s4 + e]
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const int l = 14 + 2 * s4 + e;
                Arow[(l / 3) * ldA + l % 3] = static_cast<TR>(slot(12 + e) * cond);
            }
        }
    } else {
        // slots 0..13: L[0..13]
#pragma unroll
        for (int t = 0; t < 14; ++t) Arow[(t / 3) * ldA + t % 3] = static_cast<TR>(slot(t) * cond);
    }
}

// ---- dense LU pieces (free block of the beam system in shared memory) -------------
// The pivot chains (diagonal blocks, panel solves, block back substitution)
// compute in the storage type TR: FP64 in the plain form, FP32 in the FP32
// form.  Trailing updates run on the FP64 tensor cores in both forms (FP32
// operands are exact in FP64; the result is rounded once to TR on store).

// Reciprocal of a pivot: hardware approximation refined by Newton-Raphson
// steps r <- r + r (1 - d r) (each step squares the relative error): two in
// FP64 (exact to the last bit on all tested inputs), one in FP32.
__device__ __forceinline__ double pivot_rcp(double d) {
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(d));
    r = fma(r, fma(-d, r, 1.), r);
    r = fma(r, fma(-d, r, 1.), r);
    return r;
}
__device__ __forceinline__ float pivot_rcp(float d) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(d));
    return fmaf(r, fmaf(-d, r, 1.f), r);
}

// Warp-level factorisation of the kb x kb diagonal block of the panel of
// columns [p0, p0+kb): lane r holds row p0+r; pivots broadcast by shuffles.
template <typename TR>
__device__ __forceinline__ void factor_diag(TR* A, int ldA, int m, int p0, double* rpiv, int lane,
                                            int* flag) {
    const int kb = min(kPanel, m - p0);
    TR v[kPanel];
#pragma unroll
    for (int c = 0; c < kPanel; ++c) v[c] = (lane < kb && c < kb) ? A[(p0 + lane) * ldA + p0 + c] : TR(0);
#pragma unroll
    for (int j = 0; j < kPanel; ++j) {
        if (j < kb) {
            const TR d = __shfl_sync(0xffffffffu, v[j], j);
            TR u[kPanel];
#pragma unroll
            for (int c = j + 1; c < kPanel; ++c) u[c] = __shfl_sync(0xffffffffu, v[c], j);
            const TR rp = pivot_rcp(d);
            if (lane == 0) {
                rpiv[p0 + j] = static_cast<double>(rp);
                if (!(fabs(d) > TR(0)) || !isfinite(rp)) *flag |= 2;
            }
            if (lane > j) {
                const TR l = v[j] * rp;
                v[j] = l;
#pragma unroll
                for (int c = j + 1; c < kPanel; ++c) v[c] -= l * u[c];
            }
        }
    }
    if (lane < kb) {
#pragma unroll
        for (int c = 0; c < kPanel; ++c)
            if (c < kb) A[(p0 + lane) * ldA + p0 + c] = v[c];
    }
}

// L21 = A21 U11^{-1} for rows [r_begin, m) of the panel [p0, p0+kb), rows
// strided by `stride` starting at r_begin + idx.
template <typename TR>
__device__ __forceinline__ void solve_l21(TR* A, int ldA, int m, int p0, const double* rpiv,
                                          int r_begin, int idx, int stride) {
    const int kb = min(kPanel, m - p0);
#pragma unroll 2
    for (int r = r_begin + idx; r < m; r += stride) {
        TR u[kPanel];
#pragma unroll
        for (int c = 0; c < kPanel; ++c) u[c] = (c < kb) ? A[r * ldA + p0 + c] : TR(0);
#pragma unroll
        for (int j = 0; j < kPanel; ++j) {
            if (j < kb) {
                u[j] *= static_cast<TR>(rpiv[p0 + j]);
#pragma unroll
                for (int k = j + 1; k < kPanel; ++k)
                    if (k < kb) u[k] -= u[j] * A[(p0 + j) * ldA + p0 + k];
            }
        }
#pragma unroll
        for (int c = 0; c < kPanel; ++c)
            if (c < kb) A[r * ldA + p0 + c] = u[c];
    }
}

// Warp-level factorisation of the panel of columns [p0, p0+kb): diagonal
// block, then L21 for the rows below (one row per lane per pass).
template <typename TR>
__device__ __forceinline__ void factor_panel(TR* A, int ldA, int m, int p0, double* rpiv, int lane,
                                             int* flag) {
    factor_diag(A, ldA, m, p0, rpiv, lane, flag);
    __syncwarp();
    solve_l21(A, ldA, m, p0, rpiv, p0 + min(kPanel, m - p0), lane, 32);
}

// One warp applies panel [k0, k0+kb) to the column tile [c0, c0+8) (columns
// beyond m masked) for rows [rb0, rb1): U12 = L11^{-1} A12 for the tile, then
// A22 -= L21 U12 on the FP64 tensor cores (8x8x4 tiles, two k-steps).
// Where U12 goes:
//   kU12InPlace  - lanes 0..7 solve one column each and overwrite A12 (the
//                  tile of U12 is part of the factorisation);
//   kU12ToStage  - same, but into stage[8][8]; the caller copies it into A once
//                  no other warp reads that A12 tile any more;
//   kU12InRegs   - every lane solves column c0 + lane/4 in registers and
//                  nothing is written (a helper warp on rows of a tile whose
//                  U12 another warp stores).
enum U12Mode { kU12InPlace = 0, kU12ToStage = 1, kU12InRegs = 2 };

template <int kMode, typename TR>
__device__ __forceinline__ void update_tile(TR* A, int ldA, int m, int k0, int kb, int c0, int rb0,
                                            int rb1, double* stage, int lane) {
    const int r0 = k0 + kb;
    const int s4 = lane & 3;
    const int kk0 = k0 + s4, kk1 = k0 + 4 + s4;
    double b0, b1;
    if (kMode != kU12InRegs) {
        if (lane < 8 && c0 + lane <= m) {
            const int c = c0 + lane;
            TR u[kPanel];
#pragma unroll
            for (int j = 0; j < kPanel; ++j) u[j] = (j < kb) ? A[(k0 + j) * ldA + c] : TR(0);
#pragma unroll
            for (int q = 0; q < kPanel - 1; ++q) {
#pragma unroll
                for (int j = q + 1; j < kPanel; ++j)
                    if (j < kb) u[j] -= A[(k0 + j) * ldA + k0 + q] * u[q];
            }
            if (kMode == kU12InPlace) {
#pragma unroll
                for (int j = 1; j < kPanel; ++j)
                    if (j < kb) A[(k0 + j) * ldA + c] = u[j];
            } else {
#pragma unroll
                for (int j = 0; j < kPanel; ++j) stage[j * 8 + lane] = static_cast<double>(u[j]);
            }
        }
        __syncwarp();
        const int bcol = c0 + (lane >> 2);
        const bool bok = bcol <= m;
        if (kMode == kU12InPlace) {
            b0 = (kk0 < r0 && bok) ? static_cast<double>(A[kk0 * ldA + bcol]) : 0.;
            b1 = (kk1 < r0 && bok) ? static_cast<double>(A[kk1 * ldA + bcol]) : 0.;
        } else {
            b0 = (kk0 < r0 && bok) ? stage[s4 * 8 + (lane >> 2)] : 0.;
            b1 = (kk1 < r0 && bok) ? stage[(4 + s4) * 8 + (lane >> 2)] : 0.;
        }
    } else {
        const int col = c0 + (lane >> 2);
        const bool cok = col <= m;
        TR u[kPanel];
#pragma unroll
        for (int j = 0; j < kPanel; ++j) u[j] = (j < kb && cok) ? A[(k0 + j) * ldA + (cok ? col : c0)] : TR(0);
#pragma unroll
        for (int q = 0; q < kPanel - 1; ++q) {
#pragma unroll
            for (int j = q + 1; j < kPanel; ++j)
                if (j < kb) u[j] -= A[(k0 + j) * ldA + k0 + q] * u[q];
        }
        b0 = u[0];
        b1 = u[4];
#pragma unroll
        for (int t = 1; t < 4; ++t) {
            b0 = (s4 == t) ? u[t] : b0;
            b1 = (s4 == t) ? u[4 + t] : b1;
        }
        if (kk0 >= r0) b0 = 0.;
        if (kk1 >= r0) b1 = 0.;
    }
    const int dcol = c0 + 2 * s4;
    const bool c0ok = dcol <= m, c1ok = dcol + 1 <= m;
#pragma unroll 2
    for (int rb = rb0; rb < rb1; rb += 8) {
        const int row = rb + (lane >> 2);
        const bool rv = row < rb1;
        const double a0 = (rv && kk0 < r0) ? -static_cast<double>(A[row * ldA + kk0]) : 0.;
        const double a1 = (rv && kk1 < r0) ? -static_cast<double>(A[row * ldA + kk1]) : 0.;
        double d0 = (rv && c0ok) ? static_cast<double>(A[row * ldA + dcol]) : 0.;
        double d1 = (rv && c1ok) ? static_cast<double>(A[row * ldA + dcol + 1]) : 0.;
        dmma884(d0, d1, a0, b0);
        dmma884(d0, d1, a1, b1);
        if (rv && c0ok) A[row * ldA + dcol] = static_cast<TR>(d0);
        if (rv && c1ok) A[row * ldA + dcol + 1] = static_cast<TR>(d1);
    }
}

// Solves L U y = r for the right-hand side in column rc (rows [0, m)) by one
// warp, in place, with the factors as the LU leaves them (unit L below the
// diagonal, U with its pivots on it, reciprocal pivots in rpiv): forward then
// back substitution, one column per step.
template <typename TR>
__device__ void solve_factored_column(TR* A, int ldA, int m, int rc, const double* rpiv, int lane) {
    for (int j = 0; j < m; ++j) {
        const double yj = static_cast<double>(A[j * ldA + rc]);
        for (int i = j + 1 + lane; i < m; i += 32)
            A[i * ldA + rc] = static_cast<TR>(static_cast<double>(A[i * ldA + rc]) -
                                              static_cast<double>(A[i * ldA + j]) * yj);
        __syncwarp();
    }
    for (int j = m - 1; j >= 0; --j) {
        const double yj = static_cast<double>(A[j * ldA + rc]) * rpiv[j];
        __syncwarp();
        if (lane == 0) A[j * ldA + rc] = static_cast<TR>(yj);
        for (int i = lane; i < j; i += 32)
            A[i * ldA + rc] = static_cast<TR>(static_cast<double>(A[i * ldA + rc]) -
                                              static_cast<double>(A[i * ldA + j]) * yj);
        __syncwarp();
    }
}

// Replaces the kb x kb upper-triangular diagonal block of panel p0 (pivots in
// rpiv) by its inverse; lane j < kb computes column j by back substitution
// (lanes >= kb compute on padding and store nothing).
template <typename TR>
__device__ __forceinline__ void invert_diag_block(TR* A, int ldA, int m, int p0, const double* rpiv,
                                                  int lane) {
    const int kb = min(kPanel, m - p0);
    const int jc = lane & 7;
    TR x[kPanel];
#pragma unroll
    for (int i = 0; i < kPanel; ++i) x[i] = (i == jc) ? TR(1) : TR(0);
#pragma unroll
    for (int c = kPanel - 1; c >= 0; --c) {
        if (c < kb) {  // warp-uniform; x[c] = 0 for c > jc, so no lane test is needed
            x[c] *= static_cast<TR>(rpiv[p0 + c]);
#pragma unroll
            for (int i = 0; i < c; ++i) x[i] -= A[(p0 + i) * ldA + p0 + c] * x[c];
        }
    }
    __syncwarp();
    if (lane < kb) {
#pragma unroll
        for (int i = 0; i < kPanel; ++i)
            if (i <= lane) A[(p0 + i) * ldA + p0 + lane] = x[i];
    }
}

// Block back substitution U x = y by one warp (y in column m), with the
// diagonal blocks already inverted: x_b = U_bb^{-1} y_b, then the rows above
// the block take y_i -= U_i,b x_b.  Arithmetic in TR; the solution is written
// to xs in FP64.
template <typename TR>
__device__ __forceinline__ void back_substitute_blocked(const TR* A, int ldA, int m, double* xs, int lane) {
    for (int i = lane; i < m; i += 32) xs[i] = static_cast<double>(A[i * ldA + m]);
    __syncwarp();
    const int nblk = (m + kPanel - 1) / kPanel;
    for (int b = nblk - 1; b >= 0; --b) {
        const int k0 = b * kPanel, kb = min(kPanel, m - k0);
        TR xv = TR(0);
        if (lane < kb) {
#pragma unroll
            for (int c = 0; c < kPanel; ++c)
                if (c >= lane && c < kb) xv += A[(k0 + lane) * ldA + k0 + c] * static_cast<TR>(xs[k0 + c]);
        }
        __syncwarp();
        if (lane < kb) xs[k0 + lane] = static_cast<double>(xv);
        __syncwarp();
        TR xb[kPanel];
#pragma unroll
        for (int c = 0; c < kPanel; ++c) xb[c] = (c < kb) ? static_cast<TR>(xs[k0 + c]) : TR(0);
#pragma unroll 2
        for (int i = lane; i < k0; i += 32) {
            TR acc = static_cast<TR>(xs[i]);
#pragma unroll
            for (int c = 0; c < kPanel; ++c)
                if (c < kb) acc -= A[i * ldA + k0 + c] * xb[c];
            xs[i] = static_cast<double>(acc);
        }
        __syncwarp();
    }
}

// ---- register-resident Gauss-Jordan solve of the free block ----------------------
// The free block A[0:m][0:m] and its right-hand-side columns are spread over a
// (NT/16) x 16 grid of threads: thread (ri, cj) = (tid / 16, tid % 16) keeps the
// entries (ri + a*(NT/16), cj + 16*b), a < RT, b < CT, in registers (cyclic in
// both directions, so every thread keeps work until the last pivot).  Each
// pivot step is one CTA barrier: every thread reads the pivot column and row
// from a double-buffered shared-memory slot, forms the reciprocal pivot itself
// and updates its entries; the owners of the next pivot's column and row
// publish them into the other slot.  No single warp runs a serial panel, and
// the triangular solves of an LU disappear (Gauss-Jordan eliminates above the
// pivot as well), so the chain is m steps of ~one barrier each.
// Tile sizes per (type, threads): the registers a thread can spend on the block
// within its launch budget.  Blocks that do not fit take the panel LU.
template <typename TR, int NT>
struct GJTile;
template <> struct GJTile<double, 128> { static constexpr int RT = 7, CT = 4; };
template <> struct GJTile<double, 256> { static constexpr int RT = 6, CT = 6; };
template <> struct GJTile<double, 512> { static constexpr int RT = 4, CT = 8; };
template <> struct GJTile<float, 128> { static constexpr int RT = 8, CT = 5; };
template <> struct GJTile<float, 256> { static constexpr int RT = 8, CT = 8; };
template <> struct GJTile<float, 512> { static constexpr int RT = 4, CT = 8; };

constexpr int kGJCols = 16;  // column groups of the register grid
// Largest backward error an FP64 Gauss-Jordan solve may leave (rounding gives
// ~n eps); above it the unpivoted elimination has lost accuracy to growth.
constexpr double kGJBackwardErrorMax = 1e-10;

template <typename TR, int NT>
__host__ __device__ constexpr int gj_slot() {
    return 2 * (GJTile<TR, NT>::RT * (NT / kGJCols) + GJTile<TR, NT>::CT * kGJCols);
}
static_assert(gj_slot<double, 128>() == gj_slot_entries(8, 128) &&
                  gj_slot<double, 256>() == gj_slot_entries(8, 256) &&
                  gj_slot<double, 512>() == gj_slot_entries(8, 512) &&
                  gj_slot<float, 128>() == gj_slot_entries(4, 128) &&
                  gj_slot<float, 256>() == gj_slot_entries(4, 256) &&
                  gj_slot<float, 512>() == gj_slot_entries(4, 512),
              "gj_slot_entries must follow GJTile");

// Whether the free block (m rows, m + nrhs columns; INV: m x m) fits the grid.
template <typename TR, int NT>
__host__ __device__ inline bool gj_fits(int m, int ncols) {
    return m <= GJTile<TR, NT>::RT * (NT / kGJCols) && ncols <= GJTile<TR, NT>::CT * kGJCols;
}

// Pair of TR values for vectorised shared-memory access.
template <typename TR> struct Pair2;
template <> struct Pair2<double> { using type = double2; };
template <> struct Pair2<float> { using type = float2; };

// Rank-2 update R[a][b] -= x0[a] u0[b] + x1[a] u1[b] of the column blocks
// b >= b0 (one uniform test per column block, none per entry: padding rows and
// columns hold zeros, so their updates change nothing).  (u0, u1) of column
// block b is read from the pivot pair's row buffer `rp` (pairs per column).
template <int B, typename TR, int RT, int CT>
__device__ __forceinline__ void gj_rank2_from(TR (&R)[RT][CT], const TR (&x0)[RT], const TR (&x1)[RT],
                                              const TR* rp, int b0) {
    using P2 = typename Pair2<TR>::type;
    if constexpr (B < CT) {
        if (B >= b0) {
            const P2 w = *reinterpret_cast<const P2*>(rp + 2 * B * kGJCols);
#pragma unroll
            for (int a = 0; a < RT; ++a) R[a][B] = fma(-x1[a], w.y, fma(-x0[a], w.x, R[a][B]));
        }
        gj_rank2_from<B + 1>(R, x0, x1, rp, b0);
    }
}

// Row a of R (a chosen at run time, the same in the whole warp) becomes
// p u0 + q u1 in the column blocks b >= b0, (u0, u1) from the row buffer `rp`.
template <typename TR, int RT, int CT>
__device__ __forceinline__ void gj_set_row(TR (&R)[RT][CT], int a_sel, TR p, TR q, const TR* rp, int b0) {
    using P2 = typename Pair2<TR>::type;
#pragma unroll
    for (int a = 0; a < RT; ++a)
        if (a == a_sel) {
#pragma unroll
            for (int b = 0; b < CT; ++b)
                if (b >= b0) {
                    const P2 w = *reinterpret_cast<const P2*>(rp + 2 * b * kGJCols);
                    R[a][b] = fma(p, w.x, q * w.y);
                }
        }
}

// Gauss-Jordan elimination without pivoting of the free block, held in R, two
// pivots per step (2x2 pivot blocks D, inverted through their determinant), so
// one CTA barrier serves two pivots.  Rows of a pivot pair are normalised
// (D^-1 applied), so on exit the block is the identity:
//   INV = false (solve): columns [0, m + nrhs) are loaded (only column blocks
//     that still hold a column right of the pair are updated); on exit column
//     m + r of row i holds x_i.
//   INV = true (inverse): columns [0, m) are loaded and replaced in place by
//     the inverse (pivot rows D^-1 A_K, pivot columns -A_iK D^-1, pivot block
//     D^-1).
// m must be even (free blocks are 6 per node).  buf: 2 slots of
// gj_slot<TR, NT>() entries in shared memory: the pivot pair's two columns,
// paired per row, then its two rows, paired per column; D is the pair of the
// pivot rows.  Every thread forms D^-1 and its rows' multipliers itself; the
// pivot rows' own update (multipliers ~ identity) is overwritten by their
// normalisation.  The pivot pair's block indices are the same in every
// thread, so the owners of the pivot rows and columns branch on them
// (warp-uniform) instead of selecting among their registers.  A zero or
// non-finite determinant sets bit 2 of *flag.
template <typename TR, int NT, bool INV>
__device__ __forceinline__ void gj_eliminate(const TR* A, int ldA, int m, int nrhs, TR* buf, int* flag,
                                             TR (&R)[GJTile<TR, NT>::RT][GJTile<TR, NT>::CT]) {
    using P2 = typename Pair2<TR>::type;
    constexpr int RT = GJTile<TR, NT>::RT, CT = GJTile<TR, NT>::CT;
    constexpr int PR = NT / kGJCols, PC = kGJCols;
    constexpr int SLOT = gj_slot<TR, NT>();
    constexpr int ROWS = 2 * RT * PR;
    const int tid = threadIdx.x, ri = tid / PC, cj = tid % PC;
    const int ncols = INV ? m : m + nrhs;
#pragma unroll
    for (int a = 0; a < RT; ++a) {
        const int i = ri + a * PR;
#pragma unroll
        for (int b = 0; b < CT; ++b) {
            const int j = cj + b * PC;
            R[a][b] = (i < m && j < ncols) ? A[i * ldA + j] : TR(0);
        }
    }
    // slot 0: columns 0, 1 and rows 0, 1; padding of both slots stays zero
    for (int t = tid; t < 2 * SLOT; t += NT) {
        const int e = t % SLOT;
        TR v = TR(0);
        if (t < SLOT) {
            if (e < ROWS) {
                const int i = e >> 1, h = e & 1;
                v = (i < m) ? A[i * ldA + h] : TR(0);
            } else {
                const int j = (e - ROWS) >> 1, h = (e - ROWS) & 1;
                v = (j < ncols) ? A[h * ldA + j] : TR(0);
            }
        }
        buf[t] = v;
    }
    __syncthreads();
    for (int k = 0; k < m; k += 2) {
        const TR* cb = buf + ((k >> 1) & 1) * SLOT;
        TR* nb = buf + (((k >> 1) + 1) & 1) * SLOT;
        const P2 dA = *reinterpret_cast<const P2*>(cb + 2 * k);
        const P2 dB = *reinterpret_cast<const P2*>(cb + 2 * k + 2);
        const TR det = fma(dA.x, dB.y, -(dA.y * dB.x));
        const TR rd = pivot_rcp(det);
        if (tid == 0 && (!(fabs(det) > TR(0)) || !isfinite(rd))) atomicOr(flag, 2);
        const TR i00 = dB.y * rd, i01 = -dA.y * rd, i10 = -dB.x * rd, i11 = dA.x * rd;
        TR x0[RT], x1[RT];
#pragma unroll
        for (int a = 0; a < RT; ++a) {
            const P2 c = *reinterpret_cast<const P2*>(cb + 2 * (ri + a * PR));
            x0[a] = fma(c.x, i00, c.y * i10);
            x1[a] = fma(c.x, i01, c.y * i11);
        }
        const TR* rp = cb + ROWS + 2 * cj;  // this thread's columns in the row pair
        // solve form: column blocks left of b0 hold only eliminated columns
        const int b0 = INV ? 0 : (k + 2) / PC;
        gj_rank2_from<0>(R, x0, x1, rp, b0);
        // the pivot rows: D^-1 [row k; row k+1]
        const int ak = k / PR;
        const bool r0 = ri == k % PR, r1 = ri == (k + 1) % PR;
        if (r0 || r1) gj_set_row(R, ak, r0 ? i00 : i10, r0 ? i01 : i11, rp, b0);
        if (INV) {  // the pivot columns: -A_iK D^-1, and D^-1 in the pivot rows
            const int bk = k / PC;
            const bool c0 = cj == k % PC, c1 = cj == (k + 1) % PC;
            if (c0 || c1) {
#pragma unroll
                for (int b = 0; b < CT; ++b)
                    if (b == bk) {
#pragma unroll
                        for (int a = 0; a < RT; ++a) {
                            TR v = c0 ? -x0[a] : -x1[a];
                            if (a == ak && r0) v = c0 ? i00 : i01;
                            if (a == ak && r1) v = c0 ? i10 : i11;
                            R[a][b] = v;
                        }
                    }
            }
        }
        // publish the next pair's columns and rows
        const int kn = k + 2;
        if (kn < m) {
            const int an = kn / PR, bn = kn / PC;
            const bool c0 = cj == kn % PC, c1 = cj == (kn + 1) % PC;
            if (c0 || c1) {
                TR* dst = nb + 2 * ri + (c0 ? 0 : 1);
#pragma unroll
                for (int b = 0; b < CT; ++b)
                    if (b == bn) {
#pragma unroll
                        for (int a = 0; a < RT; ++a) dst[2 * a * PR] = R[a][b];
                    }
            }
            const bool w0 = ri == kn % PR, w1 = ri == (kn + 1) % PR;
            if (w0 || w1) {
                TR* dst = nb + ROWS + 2 * cj + (w0 ? 0 : 1);
#pragma unroll
                for (int a = 0; a < RT; ++a)
                    if (a == an) {
#pragma unroll
                        for (int b = 0; b < CT; ++b) dst[2 * b * PC] = R[a][b];
                    }
            }
        }
        __syncthreads();
    }
}

// Column `col` (col >= m) of the register grid after the solve form: the
// solution for that right-hand side, into out[0:m].
template <typename TR, int NT, typename Out>
__device__ __forceinline__ void gj_extract(const TR (&R)[GJTile<TR, NT>::RT][GJTile<TR, NT>::CT], int m,
                                           int col, Out* out) {
    constexpr int RT = GJTile<TR, NT>::RT, CT = GJTile<TR, NT>::CT;
    constexpr int PR = NT / kGJCols, PC = kGJCols;
    const int tid = threadIdx.x, ri = tid / PC, cj = tid % PC;
    if (cj != col % PC) return;
    const int bc = col / PC;
#pragma unroll
    for (int b = 0; b < CT; ++b)
        if (b == bc) {
#pragma unroll
            for (int a = 0; a < RT; ++a) {
                const int i = ri + a * PR;
                if (i < m) out[i] = static_cast<Out>(R[a][b]);
            }
        }
}

// y = M v for the free block, with M either the register grid (from_regs) or
// the block in shared memory (A, FP64 accumulation in both); v, y in FP64
// shared memory.  With `bvec`, y = bvec - M v and amax gets max |y| (lane 0 of
// each row group, reduced by the caller).  The 16 threads of a row group sit
// in one half-warp and sum their columns by shuffles.
template <typename TR, int NT, bool from_regs>
__device__ __forceinline__ void gj_matvec(const TR (&R)[GJTile<TR, NT>::RT][GJTile<TR, NT>::CT], const TR* A,
                                          int ldA, int m, const double* v, const double* bvec, double* y,
                                          double& amax) {
    constexpr int RT = GJTile<TR, NT>::RT, CT = GJTile<TR, NT>::CT;
    constexpr int PR = NT / kGJCols, PC = kGJCols;
    const int tid = threadIdx.x, ri = tid / PC, cj = tid % PC;
    amax = 0.;
#pragma unroll
    for (int a = 0; a < RT; ++a) {
        const int i = ri + a * PR;
        if (a * PR >= m) break;  // uniform: no row of this block is in range
        double acc = 0.;
#pragma unroll
        for (int b = 0; b < CT; ++b) {
            const int j = cj + b * PC;
            if (j < m && i < m) {
                const double mij = from_regs ? static_cast<double>(R[a][b]) : static_cast<double>(A[i * ldA + j]);
                acc = fma(mij, v[j], acc);
            }
        }
#pragma unroll
        for (int o = 8; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (cj == 0 && i < m) {
            const double val = bvec ? bvec[i] - acc : acc;
            y[i] = val;
            amax = fmax(amax, fabs(val));
        }
    }
}

// Residual, gradient blocks and G^T lambda of one constraint on node q `nu`
// (calculate_constraint_residual_gradient.hpp:60-320 and :468-540 with
// calculate_{fixed,prescribed}_bc_constraint.hpp,
// calculate_rigid_joint_constraint.hpp:17-113 and
// calculate_rotation_control_constraint.hpp:17-144).  FixedBC: R1 = I, u1 = 0;
// PrescribedBC: (u1, R1) = the record's input; joints: (u1, R1) = the hub
// node's q `hq`, X0 = target x0 - hub x0, and the base-node blocks
// tilde(R1 X0) T_hub and -AX(C) T_hub are kept for the hub elimination.
// RotationControl puts the commanded rotation Rc = exp(angle * axis) (angle =
// input[0]) between the target and the hub: C = R(R2 Rc^-1 R1^-1).
__device__ inline void constraint_record(double* cr, int type, const double* nu, const double* X0,
                                         const double* Rt, const double* hq, const double* RtHub,
                                         const double* axis) {
    double u1[3] = {0., 0., 0.}, R1[4] = {1., 0., 0., 0.};
    if (type == KYN_CONSTRAINT_PRESCRIBED_BC) {
        for (int k = 0; k < 3; ++k) u1[k] = cr[conrec::inp + k];
        for (int k = 0; k < 4; ++k) R1[k] = cr[conrec::inp + 3 + k];
    } else if (is_hub_joint(type)) {
        for (int k = 0; k < 3; ++k) u1[k] = hq[k];
        for (int k = 0; k < 4; ++k) R1[k] = hq[3 + k];
    }
    const double len = sqrt(R1[0] * R1[0] + R1[1] * R1[1] + R1[2] * R1[2] + R1[3] * R1[3]);
    const double R1t[4] = {R1[0] / len, -R1[1] / len, -R1[2] / len, -R1[3] / len};
    double R1X0[3];
    for (int i = 0; i < 3; ++i) {
        R1X0[i] = 0.;
        for (int j = 0; j < 3; ++j) R1X0[i] += rot_entry(R1, i, j) * X0[j];
    }
    for (int i = 0; i < 3; ++i) cr[conrec::Phi + i] = nu[i] + X0[i] - u1[i] - R1X0[i];
    double R2R1t[4];
    if (type == KYN_CONSTRAINT_ROTATION_CONTROL) {
        // quaternion of the rotation vector axis*angle (quaternion_operations.hpp:231-242)
        const double ang = cr[conrec::inp];
        const double rv[3] = {axis[0] * ang, axis[1] * ang, axis[2] * ang};
        const double th = sqrt(rv[0] * rv[0] + rv[1] * rv[1] + rv[2] * rv[2]);
        const double fac = (fabs(th) < 1e-12) ? 0. : sin(th / 2.) / th;
        const double Rc[4] = {cos(th / 2.), rv[0] * fac, rv[1] * fac, rv[2] * fac};
        const double lc = sqrt(Rc[0] * Rc[0] + Rc[1] * Rc[1] + Rc[2] * Rc[2] + Rc[3] * Rc[3]);
        const double Rct[4] = {Rc[0] / lc, -Rc[1] / lc, -Rc[2] / lc, -Rc[3] / lc};
        double R2Rct[4];
        quat_compose(nu + 3, Rct, R2Rct);
        quat_compose(R2Rct, R1t, R2R1t);
    } else {
        quat_compose(nu + 3, R1t, R2R1t);
    }
    double C[9];
    for (int e = 0; e < 9; ++e) C[e] = rot_entry(R2R1t, e / 3, e % 3);
    cr[conrec::Phi + 3] = (C[7] - C[5]) / 2.;
    cr[conrec::Phi + 4] = (C[2] - C[6]) / 2.;
    cr[conrec::Phi + 5] = (C[3] - C[1]) / 2.;
    // AX(C) = tr(C)/2 I - C/2 ; grad rotational block = AX^T ; grad^T block = AX
    const double tr = (C[0] + C[4] + C[8]) / 2.;
    double AXm[9];
    for (int e = 0; e < 9; ++e) AXm[e] = -C[e] / 2. + ((e % 4 == 0) ? tr : 0.);
    for (int e = 0; e < 9; ++e) cr[conrec::AX + e] = AXm[e];
    // B rotational block = AX^T * Rt  (Rt = stored tangent block of the node)
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double acc = 0.;
            for (int k = 0; k < 3; ++k) acc += AXm[k * 3 + i] * Rt[k * 3 + j];
            cr[conrec::Brot + i * 3 + j] = acc;
        }
    // grad^T lambda
    for (int i = 0; i < 3; ++i) cr[conrec::Gl + i] = cr[conrec::lam + i];
    for (int i = 0; i < 3; ++i) {
        double acc = 0.;
        for (int k = 0; k < 3; ++k) acc += AXm[i * 3 + k] * cr[conrec::lam + 3 + k];
        cr[conrec::Gl + 3 + i] = acc;
    }
    if (is_hub_joint(type)) {
        for (int i = 0; i < 3; ++i) cr[conrec::R1X0 + i] = R1X0[i];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                double bt = 0., br = 0.;
                for (int k = 0; k < 3; ++k) {
                    bt += tilde_e(R1X0, i, k) * RtHub[k * 3 + j];
                    br -= AXm[i * 3 + k] * RtHub[k * 3 + j];
                }
                cr[conrec::Btr + i * 3 + j] = bt;
                cr[conrec::Brr + i * 3 + j] = br;
            }
    }
}

// G_base^T w of a rigid joint (base gradient [-I, tilde(R1 X0); 0, -AX]):
// [-w_t; tilde(R1 X0)^T w_t - AX^T w_r], accumulated into out.
__device__ inline void joint_base_transpose_add(const double* cr, const double* w, double* out) {
    const double* r = cr + conrec::R1X0;
    const double* AX = cr + conrec::AX;
    for (int i = 0; i < 3; ++i) out[i] -= w[i];
    for (int i = 0; i < 3; ++i) {
        double acc = 0.;
        for (int k = 0; k < 3; ++k) acc += tilde_e(r, k, i) * w[k] - AX[k * 3 + i] * w[3 + k];
        out[3 + i] += acc;
    }
}

// ---- drive train: revolute joint between hub-chain records 0 and 1 -------------------
// Residual, gradient rows and G^T lambda of the revolute joint
// (calculate_revolute_joint_constraint.hpp:19-113, calculate_revolute_joint_force.hpp:19-45,
// branch :388-465 of calculate_constraint_residual_gradient.hpp).  Rows 0-2:
// u2 + X0 - u1 - R1 X0 with gradients I (target) and -I (base); rows 3-4:
// (R2 z0).(R1 x0) and (R2 y0).(R1 x0) with gradients -(x cross z), -(x cross y)
// on the target's rotation and +(x cross z), +(x cross y) on the base's.
// `b` and `t` are hub-chain records (state at hubrec offsets).
__device__ inline void revolute_record(double* rr, const double* b, const double* t) {
    const double* X0 = t + hubrec::X0;
    const double* ax = t + hubrec::axes;
    const double* bq = b + hubrec::q;
    const double* tq = t + hubrec::q;
    double R1X0[3], x[3], y[3], z[3], ta[3];
    for (int i = 0; i < 3; ++i) {
        R1X0[i] = x[i] = y[i] = z[i] = ta[i] = 0.;
        for (int j = 0; j < 3; ++j) {
            R1X0[i] += rot_entry(bq + 3, i, j) * X0[j];
            x[i] += rot_entry(bq + 3, i, j) * ax[j];
            y[i] += rot_entry(tq + 3, i, j) * ax[3 + j];
            z[i] += rot_entry(tq + 3, i, j) * ax[6 + j];
            ta[i] += rot_entry(tq + 3, i, j) * ax[j];
        }
    }
    for (int i = 0; i < 3; ++i) rr[revrec::Phi + i] = tq[i] + X0[i] - bq[i] - R1X0[i];
    rr[revrec::Phi + 3] = z[0] * x[0] + z[1] * x[1] + z[2] * x[2];
    rr[revrec::Phi + 4] = y[0] * x[0] + y[1] * x[1] + y[2] * x[2];
    const double xcz[3] = {x[1] * z[2] - x[2] * z[1], x[2] * z[0] - x[0] * z[2], x[0] * z[1] - x[1] * z[0]};
    const double xcy[3] = {x[1] * y[2] - x[2] * y[1], x[2] * y[0] - x[0] * y[2], x[0] * y[1] - x[1] * y[0]};
    for (int i = 0; i < 3; ++i) {
        rr[revrec::x + i] = x[i];
        rr[revrec::y + i] = y[i];
        rr[revrec::z + i] = z[i];
        rr[revrec::xcz + i] = xcz[i];
        rr[revrec::xcy + i] = xcy[i];
        rr[revrec::sys + i] = ta[i] * t[hubrec::input];
    }
    // B = G T on the rotational columns (stored tangent blocks, row-major)
    const double* Tt = t + hubrec::tangent;
    const double* Tb = b + hubrec::tangent;
    for (int j = 0; j < 3; ++j) {
        double a0 = 0., a1 = 0., b0 = 0., b1 = 0.;
        for (int k = 0; k < 3; ++k) {
            a0 -= xcz[k] * Tt[k * 3 + j];
            a1 -= xcy[k] * Tt[k * 3 + j];
            b0 += xcz[k] * Tb[k * 3 + j];
            b1 += xcy[k] * Tb[k * 3 + j];
        }
        rr[revrec::Bt + j] = a0;
        rr[revrec::Bt + 3 + j] = a1;
        rr[revrec::Bb + j] = b0;
        rr[revrec::Bb + 3 + j] = b1;
    }
    const double* l = rr + revrec::lam;
    for (int i = 0; i < 3; ++i) {
        rr[revrec::GtL + i] = l[i];
        rr[revrec::GbL + i] = -l[i];
        rr[revrec::GtL + 3 + i] = -xcz[i] * l[3] - xcy[i] * l[4];
        rr[revrec::GbL + 3 + i] = xcz[i] * l[3] + xcy[i] * l[4];
    }
}

// Target correction of a six-row joint (constraint record cr, base blocks
// Btr/Brr, target block Brot) from its base correction xb: B_t x = -s Phi -
// B_base xb, with s = 1 for the correction and 0 for its part per unit shaft
// rotation.
__device__ inline bool joint_target_correction(const double* cr, const double* xb, double s, double* x) {
    double rr[3];
    for (int i = 0; i < 3; ++i) {
        x[i] = -s * cr[conrec::Phi + i] + xb[i];
        rr[i] = -s * cr[conrec::Phi + 3 + i];
        for (int k = 0; k < 3; ++k) {
            x[i] -= cr[conrec::Btr + i * 3 + k] * xb[3 + k];
            rr[i] -= cr[conrec::Brr + i * 3 + k] * xb[3 + k];
        }
    }
    return solve3(cr + conrec::Brot, rr, x + 3);
}

// Target test vector of a six-row joint from its base test vector: G_t w =
// -G_base wb with the gradients (not B = G T): G_t = [I 0; 0 AX^T],
// G_base = [-I tilde(R1 X0); 0 -AX].
__device__ inline bool joint_target_test(const double* cr, const double* wb, double* w) {
    const double* r = cr + conrec::R1X0;
    const double* AX = cr + conrec::AX;
    double rhs[3], AXt[9];
    for (int i = 0; i < 3; ++i) {
        w[i] = wb[i];
        rhs[i] = 0.;
        for (int k = 0; k < 3; ++k) {
            w[i] -= tilde_e(r, i, k) * wb[3 + k];
            rhs[i] += AX[i * 3 + k] * wb[3 + k];
            AXt[i * 3 + k] = AX[k * 3 + i];
        }
    }
    return solve3(AXt, rhs, w + 3);
}

// ---- point masses and springs at the nodes of one CTA's system ---------------------
// Adds, for local node n, the terms of every point mass at n
// (src/system/masses/calculate_quadrature_point_values.hpp:40-152: residual
// Fi - Fg, block b'Muu + g'Guu + Kuu T) and of every spring with an end at n
// (src/system/springs/calculate_quadrature_point_values.hpp:27-92: residual
// +-f, translational blocks +-a) to resid[n] and to node n's block row of A
// (scaled by the conditioner).  One thread per node: each writes only its own
// rows, and takes its elements in element order.
// Node n's rows and columns start at pos_mul * pos[n] (6 x the node's position
// in a beam system; the first-DOF map itself in a dense model).
template <typename TR>
__device__ void add_lumped_terms(int n, const double* __restrict__ rec, int n_mass, int n_spring,
                                 const double* sq, const double* sv, const double* svd,
                                 const double* sT, const double* grav, double bprime,
                                 double gprime, double cond, const int* pos, TR* A, int ldA,
                                 double* resid, int pos_mul = 6) {
    TR* Arow = A + (pos_mul * pos[n]) * ldA;
    const int cn = pos_mul * pos[n];
    for (int e = 0; e < n_mass; ++e) {
        const double* mr = rec + e * kMassRec;
        if (static_cast<int>(mr[0]) != n) continue;
        const double* ms = mr + 1;
        // Muu = diag(R, R) M* diag(R, R)^T, R = R(r o r0)
        double xr[4], R[9];
        quat_compose(sq + n * 7 + 3, mr + 37, xr);
        for (int e9 = 0; e9 < 9; ++e9) R[e9] = rot_entry(xr, e9 / 3, e9 % 3);
        double Mu[36];
        for (int bi = 0; bi < 2; ++bi)
            for (int bj = 0; bj < 2; ++bj)
                for (int i = 0; i < 3; ++i)
                    for (int j = 0; j < 3; ++j) {
                        double acc = 0.;
                        for (int k = 0; k < 3; ++k) {
                            double t = 0.;
                            for (int l = 0; l < 3; ++l) t += ms[(3 * bi + k) * 6 + 3 * bj + l] * R[j * 3 + l];
                            acc += R[i * 3 + k] * t;
                        }
                        Mu[(3 * bi + i) * 6 + 3 * bj + j] = acc;
                    }
        const double mass = Mu[0];
        const double eta[3] = {Mu[5 * 6 + 1] / mass, -Mu[5 * 6 + 0] / mass, Mu[4 * 6 + 0] / mass};
        double rho[9];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) rho[i * 3 + j] = Mu[(3 + i) * 6 + 3 + j];
        const double* ud = svd + n * 6;       // u_ddot = vd[0:3], omega_dot = vd[3:6]
        const double* od = svd + n * 6 + 3;
        const double* om = sv + n * 6 + 3;
        const double me[3] = {mass * eta[0], mass * eta[1], mass * eta[2]};
        auto mat3 = [](const double* a, const double* b, int i, int j) {
            return a[i * 3] * b[j] + a[i * 3 + 1] * b[3 + j] + a[i * 3 + 2] * b[6 + j];
        };
        double omt[9], odt[9], met[9], udt[9];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                omt[i * 3 + j] = tilde_e(om, i, j);
                odt[i * 3 + j] = tilde_e(od, i, j);
                met[i * 3 + j] = tilde_e(me, i, j);
                udt[i * 3 + j] = tilde_e(ud, i, j);
            }
        double oo[9], orho[9];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                oo[i * 3 + j] = mat3(omt, omt, i, j);
                orho[i * 3 + j] = mat3(omt, rho, i, j);
            }
        // inertial force (calculate_inertial_force.hpp) minus gravity (calculate_gravity_force.hpp)
        double r6[6];
        for (int i = 0; i < 3; ++i) {
            double acc = 0.;
            for (int k = 0; k < 3; ++k) acc += (mass * oo[i * 3 + k] + mass * odt[i * 3 + k]) * eta[k];
            r6[i] = acc + mass * ud[i] - mass * grav[i];
        }
        for (int i = 0; i < 3; ++i) {
            double acc = 0.;
            for (int k = 0; k < 3; ++k)
                acc += tilde_e(eta, i, k) * (mass * ud[k]) + rho[i * 3 + k] * od[k] + orho[i * 3 + k] * om[k] -
                       tilde_e(eta, i, k) * (mass * grav[k]);
            r6[3 + i] = acc;
        }
        for (int c = 0; c < 6; ++c) resid[n * 6 + c] += r6[c];
        // Guu (calculate_gyroscopic_matrix.hpp) and Kuu (calculate_inertia_stiffness_matrix.hpp):
        // both are zero outside the columns 3..5
        double wm[3], rw[3], rwd[3];
        for (int i = 0; i < 3; ++i) {
            wm[i] = omt[i * 3] * me[0] + omt[i * 3 + 1] * me[1] + omt[i * 3 + 2] * me[2];
            rw[i] = rho[i * 3] * om[0] + rho[i * 3 + 1] * om[1] + rho[i * 3 + 2] * om[2];
            rwd[i] = rho[i * 3] * od[0] + rho[i * 3 + 1] * od[1] + rho[i * 3 + 2] * od[2];
        }
        double G12[9], G22[9], K12[9], K22[9], M1[9];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) M1[i * 3 + j] = mat3(rho, omt, i, j) - tilde_e(rw, i, j);
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                double a12 = tilde_e(wm, j, i), k12 = 0., k22 = 0.;
                for (int k = 0; k < 3; ++k) {
                    a12 += omt[i * 3 + k] * met[j * 3 + k];
                    k12 += (odt[i * 3 + k] + oo[i * 3 + k]) * met[j * 3 + k];
                    k22 += rho[i * 3 + k] * odt[k * 3 + j] + udt[i * 3 + k] * met[k * 3 + j] +
                           omt[i * 3 + k] * M1[k * 3 + j];
                }
                G12[i * 3 + j] = a12;
                G22[i * 3 + j] = orho[i * 3 + j] - tilde_e(rw, i, j);
                K12[i * 3 + j] = k12;
                K22[i * 3 + j] = k22 - tilde_e(rwd, i, j);
            }
        // block b'Muu + g'Guu + Kuu T (T = I on the translational block)
        const double* Tn = sT + n * 9;
        for (int r = 0; r < 6; ++r) {
            for (int c = 0; c < 6; ++c) {
                double val = bprime * Mu[r * 6 + c];
                if (c >= 3) {
                    const int cc = c - 3;
                    const double* G = r < 3 ? G12 + r * 3 : G22 + (r - 3) * 3;
                    const double* K = r < 3 ? K12 + r * 3 : K22 + (r - 3) * 3;
                    val += gprime * G[cc];
                    val += K[0] * Tn[cc] + K[1] * Tn[3 + cc] + K[2] * Tn[6 + cc];
                }
                TR* a = Arow + r * ldA + cn + c;
                *a = static_cast<TR>(static_cast<double>(*a) + val * cond);
            }
        }
    }
    const double* srec = rec + n_mass * kMassRec;
    for (int e = 0; e < n_spring; ++e) {
        const double* sp = srec + e * kSpringRec;
        const int n1 = static_cast<int>(sp[0]), n2 = static_cast<int>(sp[1]);
        if (n1 != n && n2 != n) continue;
        double r[3];
        for (int c = 0; c < 3; ++c) r[c] = sp[2 + c] + sq[n2 * 7 + c] - sq[n1 * 7 + c];
        const double l = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
        const double lref = sp[5], k = sp[6];
        const double c1 = k * (lref / l - 1.);
        const double c2 = k * lref / (l * l * l);
        const double sgn = (n == n1) ? 1. : -1.;
        for (int c = 0; c < 3; ++c) resid[n * 6 + c] += sgn * (c1 * r[c]);
        const int other = (n == n1) ? n2 : n1;
        const int co = pos_mul * pos[other];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                double rr = 0.;
                for (int t = 0; t < 3; ++t) rr += tilde_e(r, i, t) * tilde_e(r, t, j);
                const double a = ((i == j) ? c1 - c2 * l * l : 0.) - c2 * rr;
                TR* d = Arow + i * ldA + cn + j;
                *d = static_cast<TR>(static_cast<double>(*d) + a * cond);
                TR* o = Arow + i * ldA + co + j;
                *o = static_cast<TR>(static_cast<double>(*o) - a * cond);
            }
    }
}

// ---- dense models: masses, springs and constraints of any row count ---------------
// A model without beam elements whose constraints are not all single-node
// six-DOF BCs (three-row constraints on position-only nodes, joints between
// its nodes) runs the reference's own bordered system in one CTA: nodes carry
// the DOFs of their freedom signature (six, or three for position-only nodes),
// constraint rows follow, and the system is solved by LU with partial
// pivoting (src/step/step.hpp:42-124 with solve_system.hpp; the order of
// operations of the dense solve follows the row-pivoting Doolittle LU).  FP64
// in both precision forms: these systems have at most kDenseModelMaxDofs unknowns.

struct DenseSmem {
    int M, b, x, q, qp, v, vd, a, qd, T, resid, con, act, fmap, red;
    // beam components (dense models with beams): shape tables, weights and
    // node state of one component at a time, its quadrature-point outputs and
    // the quadrature phase's group scratch
    int cphi, cdphi, cdphiJ, cqpw, cq, cv, cvd, cG, cFc, cFd, cgs;
    // condensed models: interior solution [6N], interior DOF map [N], the
    // bordered system's right-hand-side corrections [nd], one component's
    // local order (position of each local node, node at each position [32
    // each]) and its solution [6 cN]; M is -1 when the bordered system lives
    // in device memory (KBeam::cond_md)
    int xi, imap, bc, lpos, lnode, cx;
    int cW;  // condensed models: one component's system (inside M's region when M is shared)
    int cR;  // condensed models: bytes of that region
    int bytes;
};
// Quadrature points per pass of a condensed component's assembly.
constexpr int kCondChunk = 16;
// nt, cN, cQ: threads per CTA and the largest beam component (0: none);
// cond_nd > 0: a condensed model whose bordered system has cond_nd unknowns
// (md_global: kept in device memory instead of shared memory).
__host__ __device__ inline DenseSmem make_dense_smem(int N, int nd, int nt = 128, int cN = 0, int cQ = 0,
                                                     int cond_nd = 0, bool md_global = false) {
    DenseSmem S{};
    int o = 0;
    auto take = [&](int bytes) {
        const int r = o;
        o += (bytes + 15) & ~15;
        return r;
    };
    if (cond_nd > 0) nd = cond_nd;
    // condensed models: the bordered system's region also holds, before the
    // system is assembled, one component's system [6cN][6cN + 1], the G rows
    // of one chunk of its quadrature points, the quadrature phase's group
    // scratch and the component's tables and node state (cond_tables)
    auto r16 = [](int b) { return (b + 15) & ~15; };
    const int w_bytes = cond_nd > 0 ? r16(cN * 6 * (cN * 6 + 1) * 8) : 0;
    const int g_bytes = cond_nd > 0 ? 4 * kCondChunk * 56 * 8 : 0;
    const int s_bytes = cond_nd > 0 ? (nt / 16) * kGroupScratch * 8 : 0;
    const int t_bytes = cond_nd > 0 ? 3 * r16(cQ * cN * 8) + r16(cQ * 4 * 8) + r16(cN * 7 * 8) +
                                          2 * r16(cN * 6 * 8) + 2 * r16(cQ * 6 * 8) : 0;
    const int c_bytes = w_bytes + g_bytes + s_bytes + t_bytes;
    const int m_bytes = md_global ? 0 : nd * nd * 8;
    const int region = take(m_bytes > c_bytes ? m_bytes : c_bytes);
    S.M = md_global ? -1 : region;
    S.cW = cond_nd > 0 ? region : -1;
    S.cR = cond_nd > 0 ? (m_bytes > c_bytes ? m_bytes : c_bytes) : 0;
    S.b = take(nd * 8);
    S.x = take(nd * 8);
    S.q = take(N * 7 * 8);
    S.qp = take(N * 7 * 8);
    S.v = take(N * 6 * 8);
    S.vd = take(N * 6 * 8);
    S.a = take(N * 6 * 8);
    S.qd = take(N * 6 * 8);
    S.T = take(N * 9 * 8);
    S.resid = take(N * 6 * 8);
    S.con = take(kMaxBeamConstraints * kConStride * 8);
    S.act = take(N * 4);
    S.fmap = take(N * 4);
    S.red = take(64 * 8);  // per-warp partial sums of the error
    S.cphi = S.cdphi = S.cdphiJ = S.cqpw = S.cq = S.cv = S.cvd = S.cG = S.cFc = S.cFd = S.cgs = -1;
    if (cN > 0 && cond_nd > 0) {  // inside the bordered system's region, after the component's system
        int t = region + w_bytes;
        auto at = [&](int bytes) {
            const int r = t;
            t += r16(bytes);
            return r;
        };
        S.cG = at(g_bytes);
        S.cgs = at(s_bytes);
        S.cphi = at(cQ * cN * 8);
        S.cdphi = at(cQ * cN * 8);
        S.cdphiJ = at(cQ * cN * 8);
        S.cqpw = at(cQ * 4 * 8);
        S.cq = at(cN * 7 * 8);
        S.cv = at(cN * 6 * 8);
        S.cvd = at(cN * 6 * 8);
        S.cFc = at(cQ * 6 * 8);
        S.cFd = at(cQ * 6 * 8);
    } else if (cN > 0) {
        S.cphi = take(cQ * cN * 8);
        S.cdphi = take(cQ * cN * 8);
        S.cdphiJ = take(cQ * cN * 8);
        S.cqpw = take(cQ * 4 * 8);
        S.cq = take(cN * 7 * 8);
        S.cv = take(cN * 6 * 8);
        S.cvd = take(cN * 6 * 8);
        S.cG = take(4 * cQ * 56 * 8);
        S.cFc = take(cQ * 6 * 8);
        S.cFd = take(cQ * 6 * 8);
        S.cgs = take((nt / 16) * kGroupScratch * 8);
    }
    S.xi = S.imap = S.bc = S.lpos = S.lnode = S.cx = -1;
    if (cond_nd > 0) {
        S.xi = take(N * 6 * 8);
        S.imap = take(N * 4);
        S.bc = take(nd * 8);
        S.lpos = take(32 * 4);
        S.lnode = take(32 * 4);
        S.cx = take(cN * 6 * 8);
    }
    S.bytes = o;
    return S;
}


// Quadrature-point physics of one beam system (calculate_quadrature_point_values.hpp:
// a6-a10 of the step path): 16 threads per quadrature point, NT/16 points per
// pass.  Each stage gives every lane of a group the same formula on its own
// entries, so the half-warps run without divergence.  Inputs: shape tables
// phi / dphiJ [Q][N], weights qpw [Q][4], node state q [N][7], v, vd [N][6]
// (shared memory), the system's slab for the sections and reference frames
// (layout L).  Outputs: Fc, Fd + Fi - Fg [Q][6] and the weighted blocks of the
// integration GEMM G [4Q][56] (column layout gcol).  gscr: NT/16 groups of
// kGroupScratch doubles.  sec: the sections already staged in shared memory
// (sec_doubles(Q), slab order from x0'), or null to read them from the slab.
template <typename TG, int NT>
__device__ __forceinline__ void qp_phase(int N, int Q, const double* phi, const double* dphiJ,
                                         const double* qpw, const double* sq, const double* sv,
                                         const double* svd, const double* __restrict__ slab,
                                         const SlabLayout& L, const double* gravity, double beta_prime,
                                         double gamma_prime, double* gscr, TG* G, double* Fc, double* Fdig,
                                         const double* sec = nullptr) {
    constexpr int NG = NT / 16;
    const int tid = threadIdx.x;
    const int grp = tid >> 4;
    const int g = tid & 15;
    double* gs = gscr + grp * kGroupScratch;
    double* rn = gs + grec::rn;
    double* Rx = gs + grec::Rx;
    double* Rr = gs + grec::Rr;
    double* st = gs + grec::st;
    double* Mu = gs + grec::Mu;
    double* ms = gs + grec::ms;
    double* O12 = gs + grec::O12;
    double* Gu = gs + grec::Gu;
    double* Kk = gs + grec::Kk;
    double* fcv = gs + grec::fcv;
    double* Cu = gs + grec::Cu;
    const double* mst = gs + grec::mstar;
    const double* cst = gs + grec::cstar;
    const double* r0 = gs + grec::r0;
    const double* x0p = gs + grec::x0p;
    for (int q0 = 0; q0 < Q; q0 += NG) {
        const int qp = q0 + grp;
        const bool act = qp < Q;
        const double* ph_q = phi + qp * N;
        if (sec) {  // staged by the bulk copy: this point's entries in place
            const int qc = act ? qp : 0;
            const int o_r0 = (3 * Q + 1) & ~1;
            x0p = sec + qc * 3;
            r0 = sec + o_r0 + qc * 4;
            mst = sec + o_r0 + 4 * Q + qc * 36;
            cst = mst + 36 * Q;
        }
        if (act) {
            // stage this point's sections and reference frame from the slab
            // (read early: the loads overlap the interpolation below)
            for (int k = g; k < 79 && !sec; k += 16) {
                double v;
                if (k < 36) v = slab[L.mstar + qp * 36 + k];
                else if (k < 72) v = slab[L.cstar + qp * 36 + (k - 36)];
                else if (k < 76) v = slab[L.r0 + qp * 4 + (k - 72)];
                else v = slab[L.x0p + qp * 3 + (k - 76)];
                gs[grec::mstar + k] = v;
            }
            // this point's G rows start at zero (structural zeros, padding)
            TG* Gq = G + 4 * qp * 56;
            for (int t = g; t < 4 * 56; t += 16) Gq[t] = TG(0);
        }
        // (1) interpolation: r, u_ddot, omega, omega_dot, u', r'
        if (act) {
            for (int k = g; k < 20; k += 16) {
                // source column of node state and shape table for sum k
                const double* src = (k < 4) ? sq + 3 + k
                                  : (k < 7) ? svd + (k - 4)
                                  : (k < 10) ? sv + 3 + (k - 7)
                                  : (k < 13) ? svd + 3 + (k - 10)
                                  : (k < 16) ? sq + (k - 13)
                                             : sq + 3 + (k - 16);
                const int stride = (k < 4 || k >= 13) ? 7 : 6;
                const double* shp = (k < 13) ? ph_q : dphiJ + qp * N;
                double acc = 0.;
                for (int n = 0; n < N; ++n) acc += src[n * stride] * shp[n];
                gs[k] = acc;
            }
        }
        __syncwarp();
        if (act && g < 4) {
            const double nr = sqrt(gs[0] * gs[0] + gs[1] * gs[1] + gs[2] * gs[2] + gs[3] * gs[3]);
            rn[g] = gs[g] / nr;
        }
        __syncwarp();
        // (2) R(xr), R(r), rotational strain 2 E(r) r', s = x0' + u'
        if (act) {
            for (int k = g; k < 24; k += 16) {
                if (k < 9) {
                    double xr[4];
                    quat_compose(rn, r0, xr);
                    Rx[k] = rot_entry(xr, k / 3, k % 3);
                } else if (k < 18) {
                    Rr[k - 9] = rot_entry(rn, (k - 9) / 3, (k - 9) % 3);
                } else if (k < 21) {
                    // 2 E(r) r' with E = QuaternionDerivative (3x4)
                    const int i = k - 18;
                    const double* rp = gs + 16;
                    double e;
                    if (i == 0) e = -rn[1] * rp[0] + rn[0] * rp[1] - rn[3] * rp[2] + rn[2] * rp[3];
                    else if (i == 1) e = -rn[2] * rp[0] + rn[3] * rp[1] + rn[0] * rp[2] - rn[1] * rp[3];
                    else e = -rn[3] * rp[0] - rn[2] * rp[1] + rn[1] * rp[2] + rn[0] * rp[3];
                    st[3 + i] = 2. * e;
                } else {
                    ms[4 + (k - 21)] = x0p[k - 21] + gs[13 + (k - 21)];
                }
            }
        }
        __syncwarp();
        // (3) Muu = R M* R^T, Cuu = R C* R^T; translational strain
        if (act) {
            for (int o = g; o < 75; o += 16) {
                if (o < 72) {
                    const int e = o % 36;
                    const int i = e / 6, j = e % 6;
                    const int bi = i / 3, bj = j / 3, ii = i % 3, jj = j % 3;
                    const double* Cs = (o < 36) ? mst : cst;
                    double acc = 0.;
                    for (int pp = 0; pp < 3; ++pp) {
                        double t = 0.;
                        for (int ss = 0; ss < 3; ++ss)
                            t += Cs[(3 * bi + pp) * 6 + 3 * bj + ss] * Rx[jj * 3 + ss];
                        acc += Rx[ii * 3 + pp] * t;
                    }
                    if (o < 36) Mu[e] = acc;
                    else Cu[e] = acc;
                } else {
                    // strain[i] = x0' + u' - R(r) x0'  (calculate_strain.hpp:27-46)
                    const int i = o - 72;
                    double rx = 0.;
                    for (int j = 0; j < 3; ++j) rx += Rr[i * 3 + j] * x0p[j];
                    st[i] = x0p[i] + gs[13 + i] - rx;
                }
            }
        }
        __syncwarp();
        // (4) FC = Cuu eps (calculate_force_FC.hpp); mass and eta (CalculateEta)
        if (act && g < 6) {
            double f = 0.;
            for (int j = 0; j < 6; ++j) f += Cu[g * 6 + j] * st[j];
            fcv[g] = f;
            Fc[qp * 6 + g] = f;
        } else if (act && g == 6) {
            const double mass = Mu[0];
            ms[0] = mass;
            ms[1] = Mu[5 * 6 + 1] / mass;
            ms[2] = -Mu[5 * 6 + 0] / mass;
            ms[3] = Mu[4 * 6 + 0] / mass;
        }
        __syncwarp();
        const double* ud = gs + 4;
        const double* om = gs + 7;
        const double* omd = gs + 10;
        const double* sv3 = ms + 4;  // x0' + u'
        if (act && g < 9) {
            // (5) entry (i,j) of every 3x3 block: Ouu, Puu (calculate_Ouu/Puu.hpp),
            //     Guu (calculate_gyroscopic_matrix.hpp), Kuu
            //     (calculate_inertia_stiffness_matrix.hpp)
            const int i = g / 3, j = g % 3;
            const double mass = ms[0];
            const double meta[3] = {mass * ms[1], mass * ms[2], mass * ms[3]};
            double rw[3], rwd[3], wme[3];
            for (int r = 0; r < 3; ++r) {
                rw[r] = Mu[(3 + r) * 6 + 3] * om[0] + Mu[(3 + r) * 6 + 4] * om[1] +
                        Mu[(3 + r) * 6 + 5] * om[2];
                rwd[r] = Mu[(3 + r) * 6 + 3] * omd[0] + Mu[(3 + r) * 6 + 4] * omd[1] +
                         Mu[(3 + r) * 6 + 5] * omd[2];
            }
            cross3(om, meta, wme);
            double o12 = -tilde_e(fcv, i, j), o22 = -tilde_e(fcv + 3, i, j);
            double p21 = tilde_e(fcv, i, j), p22 = 0.;
            double g12 = -tilde_e(wme, i, j), g22 = -tilde_e(rw, i, j);
            double k12 = 0., k22 = -tilde_e(rwd, i, j);
            for (int k = 0; k < 3; ++k) {
                const double s_kj = tilde_e(sv3, k, j);
                const double s_ki = tilde_e(sv3, k, i);
                o12 += Cu[i * 6 + k] * s_kj;
                o22 += Cu[(3 + i) * 6 + k] * s_kj;
                p21 += s_ki * Cu[k * 6 + j];
                p22 += s_ki * Cu[k * 6 + 3 + j];
                const double w_ik = tilde_e(om, i, k);
                const double me_kj = tilde_e(meta, k, j);
                g12 -= w_ik * me_kj;
                g22 += w_ik * Mu[(3 + k) * 6 + 3 + j];
                double ww = 0.;
                for (int l = 0; l < 3; ++l) ww += tilde_e(om, i, l) * tilde_e(om, l, k);
                k12 -= (tilde_e(omd, i, k) + ww) * me_kj;
                k22 += Mu[(3 + i) * 6 + 3 + k] * tilde_e(omd, k, j);
                k22 += tilde_e(ud, i, k) * me_kj;
                double inner = -tilde_e(rw, k, j);
                for (int l = 0; l < 3; ++l) inner += Mu[(3 + k) * 6 + 3 + l] * tilde_e(om, l, j);
                k22 += w_ik * inner;
            }
            // G rows of this quadrature point (see the integration GEMM):
            //   4q+1: w [Puu left | Puu right | 0], 4q+3: w [0 | Ouu right | 0]
            const double w = qpw[qp * 4], wJ = qpw[qp * 4 + 2];
            TG* G1 = G + (4 * qp + 1) * 56;
            TG* G3 = G + (4 * qp + 3) * 56;
            O12[g] = o12;
            G3[gcol(18 + g)] = static_cast<TG>(w * o12);
            G3[gcol(18 + 9 + g)] = static_cast<TG>(w * o22);
            G1[gcol(9 + g)] = static_cast<TG>(w * p21);
            G1[gcol(18 + 9 + g)] = static_cast<TG>(w * p22);
            Gu[g] = g12;
            Gu[9 + g] = g22;
            G[(4 * qp) * 56 + gcol(18 + g)] = static_cast<TG>(wJ * k12);
            Kk[g] = k22;
        } else if (act && g < 15) {
            // Fd + Fi - Fe - Fg (calculate_force_FD.hpp, calculate_inertial_force.hpp,
            // calculate_gravity_force.hpp; Fe = 0)
            const int c = g - 9;
            const double mass = ms[0];
            const double eta[3] = {ms[1], ms[2], ms[3]};
            double fd = 0., fi, fgv;
            if (c < 3) {
                double wxe[3], wxwxe[3], wdxe[3];
                cross3(om, eta, wxe);
                cross3(om, wxe, wxwxe);
                cross3(omd, eta, wdxe);
                fi = mass * ud[c] + mass * (wxwxe[c] + wdxe[c]);
                fgv = mass * gravity[c];
            } else {
                const int i = c - 3;
                for (int k = 0; k < 3; ++k) fd += tilde_e(sv3, k, i) * fcv[k];
                double exu[3], rw[3], rwd[3], wxrw[3];
                cross3(eta, ud, exu);
                for (int r = 0; r < 3; ++r) {
                    rw[r] = Mu[(3 + r) * 6 + 3] * om[0] + Mu[(3 + r) * 6 + 4] * om[1] +
                            Mu[(3 + r) * 6 + 5] * om[2];
                    rwd[r] = Mu[(3 + r) * 6 + 3] * omd[0] + Mu[(3 + r) * 6 + 4] * omd[1] +
                             Mu[(3 + r) * 6 + 5] * omd[2];
                }
                cross3(om, rw, wxrw);
                fi = mass * exu[i] + rwd[i] + wxrw[i];
                const double mg[3] = {mass * gravity[0], mass * gravity[1],
                                      mass * gravity[2]};
                double exg[3];
                cross3(eta, mg, exg);
                fgv = exg[i];
            }
            Fdig[qp * 6 + c] = fd + fi - fgv;
        }
        __syncwarp();
        // (6) Quu_22 = SS^T (C11 SS - N~) joins Kuu_22; XI = beta' Muu + gamma' Guu;
        //     G rows 4q+0: wJ [XI left | XK right | XI right], 4q+2: (w/J) [Cuu]
        if (act) {
            const double wJ = qpw[qp * 4 + 2], wdJ = qpw[qp * 4 + 3];
            TG* G0 = G + (4 * qp) * 56;
            TG* G2 = G + (4 * qp + 2) * 56;
            if (g < 9) {
                const int i = g / 3, j = g % 3;
                double qv = 0.;
                for (int k = 0; k < 3; ++k) qv += tilde_e(sv3, k, i) * O12[k * 3 + j];
                G0[gcol(18 + 9 + g)] = static_cast<TG>(wJ * (Kk[g] + qv));
            }
            for (int e = g; e < 36; e += 16) {
                const int i = e / 6, j = e % 6;
                double gg = 0.;
                if (j >= 3) gg = Gu[(i < 3 ? 0 : 9) + (i % 3) * 3 + (j - 3)];
                const double xi = beta_prime * Mu[e] + gamma_prime * gg;
                const int col = (j < 3) ? i * 3 + j : 36 + i * 3 + (j - 3);
                G0[gcol(col)] = static_cast<TG>(wJ * xi);
                G2[gcol((j < 3) ? i * 3 + j : 18 + i * 3 + (j - 3))] = static_cast<TG>(wdJ * Cu[e]);
            }
        }
        __syncwarp();
    }
}

// Beam element terms of the components of a dense model (the step path's
// a5-a14 for elements whose nodes sit in a dense bordered system): for each
// component, the quadrature-point physics (qp_phase, on the component's local
// nodes), the residual (integrate_residual_vector.hpp:33-50) into resid of
// the model nodes, and SM_ij = S_ij T_j + I_ij (integrate_stiffness_matrix.hpp,
// integrate_inertia_matrix.hpp, calculate_system_matrix.hpp) times the
// conditioner added into the dense matrix Md at the nodes' DOF rows and
// columns (contribute_beams_to_sparse_matrix.hpp).  Components run one after
// the other, so shared nodes sum without races.
template <int NT>
__device__ void dense_beam_terms(const KBeam& KB, const StepCoeffs& P, const DenseSmem& S, unsigned char* smem_raw,
                                 const double* sq, const double* sv, const double* svd, const double* sT,
                                 const int* fmap, double* Md, int nd, double* resid) {
    const int tid = threadIdx.x;
    double* phi = reinterpret_cast<double*>(smem_raw + S.cphi);
    double* dphi = reinterpret_cast<double*>(smem_raw + S.cdphi);
    double* dphiJ = reinterpret_cast<double*>(smem_raw + S.cdphiJ);
    double* qpw = reinterpret_cast<double*>(smem_raw + S.cqpw);
    double* cq = reinterpret_cast<double*>(smem_raw + S.cq);
    double* cv = reinterpret_cast<double*>(smem_raw + S.cv);
    double* cvd = reinterpret_cast<double*>(smem_raw + S.cvd);
    double* G = reinterpret_cast<double*>(smem_raw + S.cG);
    double* Fc = reinterpret_cast<double*>(smem_raw + S.cFc);
    double* Fd = reinterpret_cast<double*>(smem_raw + S.cFd);
    double* gscr = reinterpret_cast<double*>(smem_raw + S.cgs);
    const double cond = P.conditioner;
    for (int ci = 0; ci < KB.n_comps; ++ci) {
        const double* hd = KB.comps + ci * kCompHead;
        const double* cs = KB.comps + static_cast<long>(hd[0]);
        const int N = static_cast<int>(hd[1]), Q = static_cast<int>(hd[2]);
        const double* node = hd + 3;  // model node of each local node
        const SlabLayout L = make_slab_layout(N, Q);
        for (int k = tid; k < Q * N; k += NT) {
            phi[k] = cs[L.phi + k];
            dphi[k] = cs[L.dphi + k];
            dphiJ[k] = cs[L.dphiJ + k];
        }
        for (int k = tid; k < Q * 4; k += NT) qpw[k] = cs[L.qpw + k];
        for (int k = tid; k < N * 7; k += NT) cq[k] = sq[static_cast<int>(node[k / 7]) * 7 + k % 7];
        for (int k = tid; k < N * 6; k += NT) {
            const int n = static_cast<int>(node[k / 6]);
            cv[k] = sv[n * 6 + k % 6];
            cvd[k] = svd[n * 6 + k % 6];
        }
        __syncthreads();
        qp_phase<double, NT>(N, Q, phi, dphiJ, qpw, cq, cv, cvd, cs, L, KB.gravity, P.beta_prime, P.gamma_prime,
                             gscr, G, Fc, Fd);
        __syncthreads();
        for (int t = tid; t < N * 6; t += NT) {
            const int n = t / 6, c = t % 6;
            double acc = 0.;
            for (int qp = 0; qp < Q; ++qp) {
                const double w = qpw[qp * 4], wJ = qpw[qp * 4 + 2];
                acc += (w * dphi[qp * N + n]) * Fc[qp * 6 + c] + (wJ * phi[qp * N + n]) * Fd[qp * 6 + c];
            }
            resid[static_cast<int>(node[n]) * 6 + c] += acc;
        }
        // one thread per (node pair, row): C_ij[r] = sum_q sum_m coef_m(i, j, q) G[4q+m]
        // with coef = (phi_i phi_j, phi_i phi'_j, phi'_i phi'_j, phi'_i phi_j)
        for (int t = tid; t < N * N * 6; t += NT) {
            const int pr = t / 6, r = t % 6;
            const int i = pr / N, j = pr % N;
            double Lr[3] = {0., 0., 0.}, RS[3] = {0., 0., 0.}, RI[3] = {0., 0., 0.};
            for (int qp = 0; qp < Q; ++qp) {
                const double pi = phi[qp * N + i], pj = phi[qp * N + j];
                const double di = dphi[qp * N + i], dj = dphi[qp * N + j];
                const double coef[4] = {pi * pj, pi * dj, di * dj, di * pj};
#pragma unroll
                for (int mm = 0; mm < 4; ++mm) {
                    const double* g = G + (4 * qp + mm) * 56;
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        Lr[c] += coef[mm] * g[gcol(r * 3 + c)];
                        RS[c] += coef[mm] * g[gcol(18 + r * 3 + c)];
                        RI[c] += coef[mm] * g[gcol(36 + r * 3 + c)];
                    }
                }
            }
            const int nj = static_cast<int>(node[j]);
            const double* Tj = sT + nj * 9;
            double* row = Md + (fmap[static_cast<int>(node[i])] + r) * nd + fmap[nj];
            for (int c = 0; c < 3; ++c) row[c] += cond * Lr[c];
            for (int c = 0; c < 3; ++c) {
                double v = RI[c];
                for (int k = 0; k < 3; ++k) v += RS[k] * Tj[k * 3 + c];
                row[3 + c] += cond * v;
            }
        }
        __syncthreads();
    }
}

// Record of a revolute joint in a dense model (constraint record layout drev;
// multipliers at conrec::lam, torque at conrec::inp): residual, the gradient
// rows B = G T on both nodes' rotations, G^T lambda and the torque about the
// target's joint axis (calculate_revolute_joint_constraint.hpp:19-113,
// calculate_revolute_joint_force.hpp:19-45, branch :388-465 of
// calculate_constraint_residual_gradient.hpp), as revolute_record computes it
// for the drive train's hub chain.  frame: x0, y0, z0 of the joint (rows).
namespace drev {
constexpr int Phi = 0;    // [5]
constexpr int Bt = 5;     // [2][3] rows 3-4 of G_target T_target (rotation)
constexpr int Bb = 11;    // [2][3] rows 3-4 of G_base T_base (rotation)
constexpr int sys = 17;   // [3] torque about R(target) x0
constexpr int GtL = 20;   // [6] G_target^T lambda
constexpr int GbL = 26;   // [6] G_base^T lambda
constexpr int xcz = 50;   // [3] x cross z
constexpr int xcy = 53;   // [3] x cross y
}  // namespace drev
__device__ inline void revolute_dense_record(double* cr, const double* bq, const double* tq, const double* frame,
                                             const double* X0, const double* Tb, const double* Tt) {
    double R1X0[3], x[3], y[3], z[3], ta[3];
    for (int i = 0; i < 3; ++i) {
        R1X0[i] = x[i] = y[i] = z[i] = ta[i] = 0.;
        for (int j = 0; j < 3; ++j) {
            R1X0[i] += rot_entry(bq + 3, i, j) * X0[j];
            x[i] += rot_entry(bq + 3, i, j) * frame[j];
            y[i] += rot_entry(tq + 3, i, j) * frame[3 + j];
            z[i] += rot_entry(tq + 3, i, j) * frame[6 + j];
            ta[i] += rot_entry(tq + 3, i, j) * frame[j];
        }
    }
    for (int i = 0; i < 3; ++i) cr[drev::Phi + i] = tq[i] + X0[i] - bq[i] - R1X0[i];
    cr[drev::Phi + 3] = z[0] * x[0] + z[1] * x[1] + z[2] * x[2];
    cr[drev::Phi + 4] = y[0] * x[0] + y[1] * x[1] + y[2] * x[2];
    const double xcz[3] = {x[1] * z[2] - x[2] * z[1], x[2] * z[0] - x[0] * z[2], x[0] * z[1] - x[1] * z[0]};
    const double xcy[3] = {x[1] * y[2] - x[2] * y[1], x[2] * y[0] - x[0] * y[2], x[0] * y[1] - x[1] * y[0]};
    const double torque = cr[conrec::inp];
    for (int i = 0; i < 3; ++i) {
        cr[drev::xcz + i] = xcz[i];
        cr[drev::xcy + i] = xcy[i];
        cr[drev::sys + i] = ta[i] * torque;
    }
    for (int j = 0; j < 3; ++j) {
        double a0 = 0., a1 = 0., b0 = 0., b1 = 0.;
        for (int k = 0; k < 3; ++k) {
            a0 -= xcz[k] * Tt[k * 3 + j];
            a1 -= xcy[k] * Tt[k * 3 + j];
            b0 += xcz[k] * Tb[k * 3 + j];
            b1 += xcy[k] * Tb[k * 3 + j];
        }
        cr[drev::Bt + j] = a0;
        cr[drev::Bt + 3 + j] = a1;
        cr[drev::Bb + j] = b0;
        cr[drev::Bb + 3 + j] = b1;
    }
    const double* l = cr + conrec::lam;
    for (int i = 0; i < 3; ++i) {
        cr[drev::GtL + i] = l[i];
        cr[drev::GbL + i] = -l[i];
        cr[drev::GtL + 3 + i] = -xcz[i] * l[3] - xcy[i] * l[4];
        cr[drev::GbL + 3 + i] = xcz[i] * l[3] + xcy[i] * l[4];
    }
}

// ---- condensed beam components of a dense model (KBeam::cond_nd > 0) -------------
// A component's local order: its interior nodes first (fmap < 0: nodes of this
// component only, without masses, springs or constraints), then its boundary
// nodes; lpos[k] = position of local node k, lnode[p] = local node at p.
// Returns the number of interior nodes.
template <int NT>
__device__ int cond_local_order(const double* node, int N, const int* fmap, int* lpos, int* lnode) {
    if (threadIdx.x == 0) {
        int o = 0;
        for (int pass = 0; pass < 2; ++pass)
            for (int k = 0; k < N; ++k)
                if ((fmap[static_cast<int>(node[k])] < 0) == (pass == 0)) {
                    lpos[k] = o;
                    lnode[o] = k;
                    ++o;
                }
    }
    int ni = 0;
    for (int k = 0; k < N; ++k) ni += fmap[static_cast<int>(node[k])] < 0;
    __syncthreads();
    return ni;
}

// Each component's system over its own local nodes, with the element terms of
// dense_beam_terms (residual, S_ij T_j + I_ij times the conditioner) taken
// kCondChunk quadrature points at a time.  The interior rows carry their
// complete right-hand side -conditioner (R - node_FX - f); the boundary
// nodes' residual goes to resid like the other nodes of the bordered system.
// Unpivoted elimination of the interior rows (the beam systems' LU) leaves in
// the boundary rows the Schur complement A_bb - A_bi A_ii^-1 A_ib and the
// right-hand-side correction -A_bi A_ii^-1 b_i.  The eliminated system is
// saved to the component's workspace for cond_add_schur and
// cond_back_substitute.  This is the static condensation of the element
// groups that the reference's sparse direct solve factors as one matrix
// (src/solver/compute_system_row_entries.hpp:83-97 gives their overlap).
template <int NT>
__device__ void cond_component_terms(const KBeam& KB, const StepCoeffs& P, const DenseSmem& S,
                                     unsigned char* smem_raw, const double* sq, const double* sv,
                                     const double* svd, const double* sT, const int* fmap,
                                     const double* mslab, const SlabLayout& ML, double* resid, int* flag,
                                     unsigned long long* ph = nullptr) {
    const int tid = threadIdx.x;
    // optional sub-phase timers (thread 0): quadrature physics, assembly,
    // elimination, save, in the slots kPhaseQuadrature, kPhaseLUDiag,
    // kPhaseLUPanel, kPhaseIntEpilogue of ph
    long long pt = (ph && tid == 0) ? clock64() : 0;
    auto sub = [&](int slot) {
        if (ph && tid == 0) {
            const long long t = clock64();
            ph[slot] += static_cast<unsigned long long>(t - pt);
            pt = t;
        }
    };
    double* phi = reinterpret_cast<double*>(smem_raw + S.cphi);
    double* dphi = reinterpret_cast<double*>(smem_raw + S.cdphi);
    double* dphiJ = reinterpret_cast<double*>(smem_raw + S.cdphiJ);
    double* qpw = reinterpret_cast<double*>(smem_raw + S.cqpw);
    double* cq = reinterpret_cast<double*>(smem_raw + S.cq);
    double* cv = reinterpret_cast<double*>(smem_raw + S.cv);
    double* cvd = reinterpret_cast<double*>(smem_raw + S.cvd);
    double* G = reinterpret_cast<double*>(smem_raw + S.cG);
    double* Fc = reinterpret_cast<double*>(smem_raw + S.cFc);
    double* Fd = reinterpret_cast<double*>(smem_raw + S.cFd);
    double* gscr = reinterpret_cast<double*>(smem_raw + S.cgs);
    double* W = reinterpret_cast<double*>(smem_raw + S.cW);
    int* lpos = reinterpret_cast<int*>(smem_raw + S.lpos);
    int* lnode = reinterpret_cast<int*>(smem_raw + S.lnode);
    const double cond = P.conditioner;
    for (int ci = 0; ci < KB.n_comps; ++ci) {
        const double* hd = KB.comps + ci * kCompHead;
        const double* cs = KB.comps + static_cast<long>(hd[0]);
        double* work = const_cast<double*>(KB.comps) + static_cast<long>(hd[kCompWork]);
        const int N = static_cast<int>(hd[1]), Q = static_cast<int>(hd[2]);
        const double* node = hd + 3;
        const SlabLayout L = make_slab_layout(N, Q);
        const int mc = 6 * N, ldw = mc + 1;
        for (int k = tid; k < Q * N; k += NT) {
            phi[k] = cs[L.phi + k];
            dphi[k] = cs[L.dphi + k];
            dphiJ[k] = cs[L.dphiJ + k];
        }
        for (int k = tid; k < Q * 4; k += NT) qpw[k] = cs[L.qpw + k];
        for (int k = tid; k < N * 7; k += NT) cq[k] = sq[static_cast<int>(node[k / 7]) * 7 + k % 7];
        for (int k = tid; k < N * 6; k += NT) {
            const int n = static_cast<int>(node[k / 6]);
            cv[k] = sv[n * 6 + k % 6];
            cvd[k] = svd[n * 6 + k % 6];
        }
        const int mi = 6 * cond_local_order<NT>(node, N, fmap, lpos, lnode);
        for (int k = tid; k < mc * ldw; k += NT) {
            const int r = k / ldw, c = k % ldw;
            double v = 0.;
            if (c == mc && r < mi) {  // interior right-hand side before the element residual
                const int n = static_cast<int>(node[lnode[r / 6]]) * 6 + r % 6;
                v = cond * (mslab[ML.fx + n] + mslab[ML.f + n]);
            }
            W[k] = v;
        }
        __syncthreads();
        for (int q0 = 0; q0 < Q; q0 += kCondChunk) {
            const int qn = min(kCondChunk, Q - q0);
            SlabLayout Lc = L;
            Lc.mstar += 36 * q0;
            Lc.cstar += 36 * q0;
            Lc.r0 += 4 * q0;
            Lc.x0p += 3 * q0;
            qp_phase<double, NT>(N, qn, phi + q0 * N, dphiJ + q0 * N, qpw + q0 * 4, cq, cv, cvd, cs, Lc,
                                 KB.gravity, P.beta_prime, P.gamma_prime, gscr, G, Fc, Fd);
            __syncthreads();
            sub(kPhaseQuadrature);
            for (int t = tid; t < N * 6; t += NT) {
                const int n = t / 6, c = t % 6;
                double acc = 0.;
                for (int qp = 0; qp < qn; ++qp) {
                    const int qa = q0 + qp;
                    const double w = qpw[qa * 4], wJ = qpw[qa * 4 + 2];
                    acc += (w * dphi[qa * N + n]) * Fc[qp * 6 + c] + (wJ * phi[qa * N + n]) * Fd[qp * 6 + c];
                }
                const int mn = static_cast<int>(node[n]);
                if (fmap[mn] < 0) W[(lpos[n] * 6 + c) * ldw + mc] -= cond * acc;
                else resid[mn * 6 + c] += acc;
            }
            for (int t = tid; t < N * N * 6; t += NT) {
                const int pr = t / 6, r = t % 6;
                const int i = pr / N, j = pr % N;
                double Lr[3] = {0., 0., 0.}, RS[3] = {0., 0., 0.}, RI[3] = {0., 0., 0.};
                for (int qp = 0; qp < qn; ++qp) {
                    const int qa = q0 + qp;
                    const double pi = phi[qa * N + i], pj = phi[qa * N + j];
                    const double di = dphi[qa * N + i], dj = dphi[qa * N + j];
                    const double coef[4] = {pi * pj, pi * dj, di * dj, di * pj};
#pragma unroll
                    for (int mm = 0; mm < 4; ++mm) {
                        const double* g = G + (4 * qp + mm) * 56;
#pragma unroll
                        for (int c = 0; c < 3; ++c) {
                            Lr[c] += coef[mm] * g[gcol(r * 3 + c)];
                            RS[c] += coef[mm] * g[gcol(18 + r * 3 + c)];
                            RI[c] += coef[mm] * g[gcol(36 + r * 3 + c)];
                        }
                    }
                }
                const double* Tj = sT + static_cast<int>(node[j]) * 9;
                double* row = W + (lpos[i] * 6 + r) * ldw + lpos[j] * 6;
                for (int c = 0; c < 3; ++c) row[c] += cond * Lr[c];
                for (int c = 0; c < 3; ++c) {
                    double v = RI[c];
                    for (int k = 0; k < 3; ++k) v += RS[k] * Tj[k * 3 + c];
                    row[3 + c] += cond * v;
                }
            }
            __syncthreads();
            sub(kPhaseLUDiag);
        }
        // unpivoted elimination of the interior rows, right-hand side included:
        // rows over the warps, columns over the lanes, one barrier per pivot
        // (each row's warp stores its own multiplier after using it)
        const int wid = tid >> 5, wl = tid & 31;
        for (int k = 0; k < mi; ++k) {
            const double d = W[k * ldw + k];
            if (tid == 0 && !(fabs(d) > 0. && isfinite(d))) *flag |= 2;
            const double rd = 1. / d;
            for (int i = k + 1 + wid; i < mc; i += NT / 32) {
                const double l = W[i * ldw + k] * rd;
                for (int j = k + 1 + wl; j <= mc; j += 32) W[i * ldw + j] -= l * W[k * ldw + j];
                __syncwarp();
                if (wl == 0) W[i * ldw + k] = l;
            }
            __syncthreads();
        }
        sub(kPhaseLUPanel);
        for (int k = tid; k < mc * ldw; k += NT) work[k] = W[k];
        __syncthreads();
        sub(kPhaseIntEpilogue);
    }
}

// Adds each condensed component's Schur complement (its workspace rows and
// columns of the boundary nodes) into the bordered system Md and its
// right-hand-side correction into bc, at the boundary nodes' DOF rows.
template <int NT>
__device__ void cond_add_schur(const KBeam& KB, const DenseSmem& S, unsigned char* smem_raw, const int* fmap,
                               double* Md, int md, double* bc) {
    const int tid = threadIdx.x;
    int* lpos = reinterpret_cast<int*>(smem_raw + S.lpos);
    int* lnode = reinterpret_cast<int*>(smem_raw + S.lnode);
    for (int ci = 0; ci < KB.n_comps; ++ci) {
        const double* hd = KB.comps + ci * kCompHead;
        const double* work = KB.comps + static_cast<long>(hd[kCompWork]);
        const int N = static_cast<int>(hd[1]);
        const double* node = hd + 3;
        const int mc = 6 * N, ldw = mc + 1;
        const int mi = 6 * cond_local_order<NT>(node, N, fmap, lpos, lnode);
        const int mb = mc - mi;
        for (int e = tid; e < mb * (mb + 1); e += NT) {
            const int t = mi + e / (mb + 1), u = mi + e % (mb + 1);
            const int rt = fmap[static_cast<int>(node[lnode[t / 6]])] + t % 6;
            const double v = work[t * ldw + u];
            if (u == mc) bc[rt] += v;
            else Md[rt * md + fmap[static_cast<int>(node[lnode[u / 6]])] + u % 6] += v;
        }
        __syncthreads();
    }
}

// The back substitution of cond_back_substitute for all components at once,
// one warp per component, when every component's eliminated rows and a map
// of its DOFs fit the condensed region (dead once the bordered system is
// solved): the rows are staged there together, map[p] is the position of local
// DOF p in xi (>= 0, interior) or -1 - its position in x (boundary), and each
// warp sweeps its rows with the sums of the sequential form.  Returns false,
// having done nothing, when they do not fit.
template <int NT>
__device__ bool cond_back_substitute_warps(const KBeam& KB, const DenseSmem& S, unsigned char* smem_raw,
                                           const int* fmap, const int* imap, const double* x, double* xi) {
    constexpr int NW = NT / 32;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    long need = 0;
    for (int ci = 0; ci < KB.n_comps; ++ci) {
        const int N = static_cast<int>(KB.comps[ci * kCompHead + 1]);
        int ni = 0;
        for (int k = 0; k < N; ++k) ni += fmap[static_cast<int>(KB.comps[ci * kCompHead + 3 + k])] < 0;
        need += 8L * (6 * ni) * (6 * N + 1) + 4L * 6 * N + 16;
    }
    if (need > S.cR) return false;
    unsigned char* base = smem_raw + S.cW;
    // per component: rows at a double offset, map at an int offset (tid 0 lays them out)
    __shared__ int s_roff[kMaxDenseComps], s_moff[kMaxDenseComps], s_mi[kMaxDenseComps];
    if (tid == 0) {
        long o = 0;
        for (int ci = 0; ci < KB.n_comps; ++ci) {
            const double* hd = KB.comps + ci * kCompHead;
            const int N = static_cast<int>(hd[1]), mc = 6 * N;
            int ni = 0;
            for (int k = 0; k < N; ++k) ni += fmap[static_cast<int>(hd[3 + k])] < 0;
            s_roff[ci] = static_cast<int>(o / 8);
            s_mi[ci] = 6 * ni;
            o += 8L * (6 * ni) * (mc + 1);
            s_moff[ci] = static_cast<int>(o / 4);
            int* map = reinterpret_cast<int*>(base) + s_moff[ci];
            int pi = 0, pb = 6 * ni;  // interior nodes first, then boundary, in local order
            for (int k = 0; k < N; ++k) {
                const int n = static_cast<int>(hd[3 + k]);
                if (fmap[n] < 0)
                    for (int c = 0; c < 6; ++c) map[pi++] = imap[n] + c;
                else
                    for (int c = 0; c < 6; ++c) map[pb++] = -1 - (fmap[n] + c);
            }
            o += 4L * mc;
            o = (o + 15) & ~15L;
        }
    }
    __syncthreads();
    for (int ci = 0; ci < KB.n_comps; ++ci) {
        const double* hd = KB.comps + ci * kCompHead;
        const double* work = KB.comps + static_cast<long>(hd[kCompWork]);
        const int ldw = 6 * static_cast<int>(hd[1]) + 1;
        double* R = reinterpret_cast<double*>(base) + s_roff[ci];
        for (int k = tid; k < s_mi[ci] * ldw; k += NT) R[k] = work[k];
    }
    __syncthreads();
    for (int ci = warp; ci < KB.n_comps; ci += NW) {
        const int mc = 6 * static_cast<int>(KB.comps[ci * kCompHead + 1]), ldw = mc + 1, mi = s_mi[ci];
        const double* R = reinterpret_cast<const double*>(base) + s_roff[ci];
        const int* map = reinterpret_cast<const int*>(base) + s_moff[ci];
        for (int k = mi - 1; k >= 0; --k) {
            const double* row = R + k * ldw;
            double acc = 0.;
            for (int j = k + 1 + lane; j < mc; j += 32) {
                const int mj = map[j];
                acc += row[j] * (mj >= 0 ? xi[mj] : x[-1 - mj]);
            }
            for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
            if (lane == 0) xi[map[k]] = (row[mc] - acc) / row[k];
            __syncwarp();
        }
    }
    __syncthreads();
    return true;
}

// Interior corrections of each condensed component from the bordered
// system's solution x at its boundary nodes: U_ii x_i = y_i - U_ib x_b by one
// warp, rows of the eliminated system (staged back into shared memory in W)
// from the last up; the corrections go to xi at the nodes' interior DOFs.
template <int NT>
__device__ void cond_back_substitute(const KBeam& KB, const DenseSmem& S, unsigned char* smem_raw,
                                     const int* fmap, const int* imap, const double* x, double* xi) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (cond_back_substitute_warps<NT>(KB, S, smem_raw, fmap, imap, x, xi)) return;
    double* W = reinterpret_cast<double*>(smem_raw + S.cW);
    double* cx = reinterpret_cast<double*>(smem_raw + S.cx);
    int* lpos = reinterpret_cast<int*>(smem_raw + S.lpos);
    int* lnode = reinterpret_cast<int*>(smem_raw + S.lnode);
    for (int ci = 0; ci < KB.n_comps; ++ci) {
        const double* hd = KB.comps + ci * kCompHead;
        const double* work = KB.comps + static_cast<long>(hd[kCompWork]);
        const int N = static_cast<int>(hd[1]);
        const double* node = hd + 3;
        const int mc = 6 * N, ldw = mc + 1;
        const int mi = 6 * cond_local_order<NT>(node, N, fmap, lpos, lnode);
        for (int k = tid; k < mi * ldw; k += NT) W[k] = work[k];
        for (int p = mi + tid; p < mc; p += NT) cx[p] = x[fmap[static_cast<int>(node[lnode[p / 6]])] + p % 6];
        __syncthreads();
        if (warp == 0) {
            for (int k = mi - 1; k >= 0; --k) {
                const double* row = W + k * ldw;
                double acc = 0.;
                for (int j = k + 1 + lane; j < mc; j += 32) acc += row[j] * cx[j];
                for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
                if (lane == 0) cx[k] = (row[mc] - acc) / row[k];
                __syncwarp();
            }
        }
        __syncthreads();
        for (int p = tid; p < mi; p += NT) xi[imap[static_cast<int>(node[lnode[p / 6]])] + p % 6] = cx[p];
        __syncthreads();
    }
}

template <int NT>
__device__ __forceinline__ void dense_model_step(const KBeam& KB, const StepCoeffs& P, int record, int* status_out,
                                 int* iters_out, unsigned char* smem_raw) {
    constexpr int NW = NT / 32;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int N = KB.N, nc = KB.nc;
    const SlabLayout L = make_slab_layout(N, 0);
    double* __restrict__ slab = KB.slab;
    const int nd = KB.model_dofs;                       // the reference's unknowns
    const bool cnd = KB.cond_nd > 0;                    // condensed beam components
    const int md = cnd ? KB.cond_nd : nd;               // unknowns of the bordered system
    const DenseSmem S = make_dense_smem(N, nd, NT, KB.n_comps > 0 ? KB.comp_maxN : 0, KB.comp_maxQ, KB.cond_nd,
                                        KB.cond_md != nullptr);
    double* Md = KB.cond_md ? KB.cond_md : reinterpret_cast<double*>(smem_raw + S.M);
    double* b = reinterpret_cast<double*>(smem_raw + S.b);
    double* x = reinterpret_cast<double*>(smem_raw + S.x);
    double* sq = reinterpret_cast<double*>(smem_raw + S.q);
    double* sqp = reinterpret_cast<double*>(smem_raw + S.qp);
    double* sv = reinterpret_cast<double*>(smem_raw + S.v);
    double* svd = reinterpret_cast<double*>(smem_raw + S.vd);
    double* sa = reinterpret_cast<double*>(smem_raw + S.a);
    double* sqd = reinterpret_cast<double*>(smem_raw + S.qd);
    double* sT = reinterpret_cast<double*>(smem_raw + S.T);
    double* resid = reinterpret_cast<double*>(smem_raw + S.resid);
    double* con = reinterpret_cast<double*>(smem_raw + S.con);
    int* act = reinterpret_cast<int*>(smem_raw + S.act);
    int* fmap = reinterpret_cast<int*>(smem_raw + S.fmap);
    double* red = reinterpret_cast<double*>(smem_raw + S.red);
    double* xi = cnd ? reinterpret_cast<double*>(smem_raw + S.xi) : nullptr;
    int* imap = cnd ? reinterpret_cast<int*>(smem_raw + S.imap) : nullptr;
    double* bc = cnd ? reinterpret_cast<double*>(smem_raw + S.bc) : nullptr;
    __shared__ int s_flag, s_nsys, s_piv;
    // phase timers (KYN_OPT_PHASE_TIMING): one CTA's clock, thread 0
    __shared__ unsigned long long s_ph[kNumPhases];
    const bool timing = KB.prof != nullptr;
    long long ph_t = 0;
    if (timing && tid == 0) {
        for (int k = 0; k < kNumPhases; ++k) s_ph[k] = 0ull;
        ph_t = clock64();
    }
    auto mark = [&](int phase) {
        if (timing && tid == 0) {
            const long long t = clock64();
            s_ph[phase] += static_cast<unsigned long long>(t - ph_t);
            ph_t = t;
        }
    };
    const double h = P.h;

    // state, constraint inputs, multipliers reset (ResetConstraints)
    for (int k = tid; k < N * 7; k += NT) sq[k] = slab[L.q + k];
    for (int k = tid; k < N * 6; k += NT) {
        sv[k] = slab[L.v + k];
        svd[k] = slab[L.vd + k];
        sa[k] = slab[L.a + k];
    }
    if (tid < nc) {
        double* c = con + tid * kConStride;
        for (int k = 0; k < 7; ++k) c[conrec::inp + k] = slab[L.con_input + tid * 7 + k];
        for (int k = 0; k < 6; ++k) c[conrec::lam + k] = 0.;
    }
    if (tid == 0) {
        // FreedomSignature per node (assemble_node_freedom_allocation_table.hpp):
        // masses six, springs position only, constraint targets six or three,
        // joint bases six; DOF map = exclusive scan (compute_node_freedom_map_table.hpp)
        for (int n = 0; n < N; ++n) act[n] = 0;
        if (cnd)
            for (int n = 0; n < N; ++n) imap[n] = 0;
        const double* mrec = KB.lumped;
        for (int e = 0; e < KB.n_mass; ++e) act[static_cast<int>(mrec[e * kMassRec])] |= kSigAll;
        const double* srec = KB.lumped + KB.n_mass * kMassRec;
        for (int e = 0; e < KB.n_spring; ++e) {
            act[static_cast<int>(srec[e * kSpringRec])] |= kSigPosition;
            act[static_cast<int>(srec[e * kSpringRec + 1])] |= kSigPosition;
        }
        for (int c = 0; c < nc; ++c) {
            const int t = KB.con_type[c];
            act[KB.con_node[c]] |= (t >= KYN_CONSTRAINT_FIXED_BC_3DOF) ? kSigPosition : kSigAll;
            if (KB.con_base[c] >= 0) act[KB.con_base[c]] |= kSigAll;
        }
        // condensed models: a node of one component only, with no mass, spring
        // or constraint, is interior (fmap -1, imap its first interior DOF)
        if (cnd)
            for (int n = 0; n < N; ++n) fmap[n] = act[n];
        for (int ci = 0; ci < KB.n_comps; ++ci) {  // beam nodes: all six components
            const double* hd = KB.comps + ci * kCompHead;
            for (int k = 0; k < static_cast<int>(hd[1]); ++k) {
                act[static_cast<int>(hd[3 + k])] |= kSigAll;
                if (cnd) ++imap[static_cast<int>(hd[3 + k])];
            }
        }
        int o = 0, oi = 0;
        for (int n = 0; n < N; ++n) {
            act[n] = (act[n] == kSigAll) ? 6 : (act[n] == kSigPosition) ? 3 : 0;
            if (cnd && imap[n] == 1 && fmap[n] == 0) {
                fmap[n] = -1;
                imap[n] = oi;
                oi += act[n];
            } else {
                fmap[n] = o;
                if (cnd) imap[n] = -1;
                o += act[n];
            }
        }
        int rows = 0;
        for (int c = 0; c < nc; ++c) rows += constraint_rows(KB.con_type[c]);
        s_nsys = o;
        s_flag = cnd ? ((o + rows != md || o + oi + rows != nd) ? 2 : 0) : (o > nd) ? 2 : 0;
    }
    __syncthreads();
    const int nsys = s_nsys;
    // PredictNextState (src/step/predict_next_state.hpp:14-47)
    for (int k = tid; k < N * 7; k += NT) sqp[k] = sq[k];
    for (int k = tid; k < N * 6; k += NT) {
        const double v_p = sv[k], vd_p = svd[k], a_p = sa[k];
        svd[k] = 0.;
        const double an = (P.alpha_f * vd_p - P.alpha_m * a_p) / (1. - P.alpha_m);
        sa[k] = an;
        sv[k] = v_p + h * (1. - P.gamma) * a_p + P.gamma * h * an;
        sqd[k] = v_p + (0.5 - P.beta) * h * a_p + P.beta * h * an;
    }
    __syncthreads();
    auto displacement = [&]() {
        for (int n = tid; n < N; n += NT) {
            for (int c = 0; c < 3; ++c) sq[n * 7 + c] = sqp[n * 7 + c] + h * sqd[n * 6 + c];
            const double d[3] = {h * sqd[n * 6 + 3], h * sqd[n * 6 + 4], h * sqd[n * 6 + 5]};
            double qd4[4], qn[4];
            rotvec_to_quat(d, qd4);
            quat_compose(qd4, sqp + n * 7 + 3, qn);
            for (int c = 0; c < 4; ++c) sq[n * 7 + 3 + c] = qn[c];
        }
    };
    displacement();
    __syncthreads();

    int status = KYN_NOT_CONVERGED, iters = 0;
    const double cond = P.conditioner;
    for (int iter = 0; iter < P.max_iter && s_flag == 0; ++iter) {
        // tangent operator, rotational block (src/system/calculate_tangent_operator.hpp)
        for (int n = tid; n < N; n += NT) {
            const double rv[3] = {h * sqd[n * 6 + 3], h * sqd[n * 6 + 4], h * sqd[n * 6 + 5]};
            const double ph = sqrt(rv[0] * rv[0] + rv[1] * rv[1] + rv[2] * rv[2]);
            double sn, cs;
            sincos(ph, &sn, &cs);
            const double t1 = (ph > 1.e-16) ? (cs - 1.) / (ph * ph) : 0.;
            const double t2 = (ph > 1.e-16) ? (1. - sn / ph) / (ph * ph) : 0.;
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) {
                    double rr = 0.;
                    for (int k = 0; k < 3; ++k) rr += tilde_e(rv, j, k) * tilde_e(rv, k, i);
                    sT[n * 9 + i * 3 + j] = (i == j ? 1. : 0.) + (t1 * tilde_e(rv, j, i) + t2 * rr);
                }
        }
        for (int k = tid; k < N * 6; k += NT) resid[k] = 0.;
        mark(kPhaseLoadPredict);
        if (cnd) {  // components first: their systems share the bordered system's region
            __syncthreads();
            cond_component_terms<NT>(KB, P, S, smem_raw, sq, sv, svd, sT, fmap, slab, L, resid, &s_flag,
                                     timing ? s_ph : nullptr);
        }
        mark(kPhaseIntegrate);
        for (int k = tid; k < md * md; k += NT) Md[k] = 0.;
        for (int k = tid; k < md; k += NT) b[k] = 0.;
        if (cnd)
            for (int k = tid; k < md; k += NT) bc[k] = 0.;
        __syncthreads();
        // masses and springs (residual into resid, conditioned blocks into Md)
        for (int n = tid; n < N; n += NT)
            add_lumped_terms(n, KB.lumped, KB.n_mass, KB.n_spring, sq, sv, svd, sT, KB.gravity,
                             P.beta_prime, P.gamma_prime, cond, fmap, Md, md, resid, 1);
        if (KB.n_comps > 0) {  // beam elements, then their node_FX (summed per node)
            __syncthreads();
            if (cnd) cond_add_schur<NT>(KB, S, smem_raw, fmap, Md, md, bc);
            else dense_beam_terms<NT>(KB, P, S, smem_raw, sq, sv, svd, sT, fmap, Md, nd, resid);
            for (int t = tid; t < N * 6; t += NT) resid[t] -= slab[L.fx + t];
        }
        // constraints: residual, gradients and G^T lambda
        if (tid < nc) {
            double* cr = con + tid * kConStride;
            const int t = KB.con_type[tid], tn = KB.con_node[tid], bn = KB.con_base[tid];
            if (t >= KYN_CONSTRAINT_FIXED_BC_3DOF) {
                // three rows (calculate_*_3DOF_constraint.hpp): u2 + X0 - u1 - R1 X0
                double u1[3] = {0., 0., 0.}, R1[4] = {1., 0., 0., 0.};
                if (t == KYN_CONSTRAINT_PRESCRIBED_BC_3DOF) {
                    for (int k = 0; k < 3; ++k) u1[k] = cr[conrec::inp + k];
                    for (int k = 0; k < 4; ++k) R1[k] = cr[conrec::inp + 3 + k];
                } else if (t == KYN_CONSTRAINT_RIGID_JOINT_6DOF_TO_3DOF) {
                    for (int k = 0; k < 3; ++k) u1[k] = sq[bn * 7 + k];
                    for (int k = 0; k < 4; ++k) R1[k] = sq[bn * 7 + 3 + k];
                }
                const double* X0 = KB.con_X0[tid];
                double r1x0[3];
                for (int i = 0; i < 3; ++i) {
                    r1x0[i] = 0.;
                    for (int j = 0; j < 3; ++j) r1x0[i] += rot_entry(R1, i, j) * X0[j];
                }
                for (int i = 0; i < 3; ++i) {
                    cr[conrec::Phi + i] = sq[tn * 7 + i] + X0[i] - u1[i] - r1x0[i];
                    cr[conrec::Gl + i] = cr[conrec::lam + i];
                    cr[conrec::R1X0 + i] = r1x0[i];
                }
                if (t == KYN_CONSTRAINT_RIGID_JOINT_6DOF_TO_3DOF)  // base block tilde(R1 X0) T_base
                    for (int i = 0; i < 3; ++i)
                        for (int j = 0; j < 3; ++j) {
                            double bt = 0.;
                            for (int k = 0; k < 3; ++k) bt += tilde_e(r1x0, i, k) * sT[bn * 9 + k * 3 + j];
                            cr[conrec::Btr + i * 3 + j] = bt;
                        }
            } else if (t == KYN_CONSTRAINT_REVOLUTE_JOINT) {
                revolute_dense_record(cr, sq + bn * 7, sq + tn * 7, KB.con_frames + tid * 9, KB.con_X0[tid],
                                      sT + bn * 9, sT + tn * 9);
            } else {
                constraint_record(cr, t, sq + tn * 7, KB.con_X0[tid], sT + tn * 9,
                                  bn >= 0 ? sq + bn * 7 : nullptr, bn >= 0 ? sT + bn * 9 : nullptr,
                                  KB.con_axis[tid]);
            }
        }
        __syncthreads();
        // scatter: rows of B = G T, columns G^T, residuals (assemble_constraints_matrix.hpp,
        // assemble_constraints_residual.hpp, assemble_system_residual.hpp)
        if (tid == 0) {
            int rf = nsys;
            for (int c = 0; c < nc; ++c) {
                const double* cr = con + c * kConStride;
                const int t = KB.con_type[c], tn = KB.con_node[c], bn = KB.con_base[c];
                const int rows = constraint_rows(t);
                const int ft = fmap[tn];
                if (t == KYN_CONSTRAINT_REVOLUTE_JOINT) {  // five rows, gradients on both nodes
                    const int fb = fmap[bn];
                    for (int r = 0; r < 5; ++r) {
                        double* row = Md + (rf + r) * md;
                        if (r < 3) {
                            row[ft + r] += 1.;
                            Md[(ft + r) * md + rf + r] += 1.;
                            row[fb + r] -= 1.;
                            Md[(fb + r) * md + rf + r] -= 1.;
                        } else {
                            const double* v = cr + (r == 3 ? drev::xcz : drev::xcy);
                            for (int j = 0; j < 3; ++j) {
                                row[ft + 3 + j] += cr[drev::Bt + (r - 3) * 3 + j];
                                row[fb + 3 + j] += cr[drev::Bb + (r - 3) * 3 + j];
                                Md[(ft + 3 + j) * md + rf + r] -= v[j];
                                Md[(fb + 3 + j) * md + rf + r] += v[j];
                            }
                        }
                        b[rf + r] += cr[drev::Phi + r];
                    }
                    for (int e = 0; e < 6; ++e) {
                        b[ft + e] += cr[drev::GtL + e] + (e >= 3 ? cr[drev::sys + e - 3] : 0.);
                        b[fb + e] += cr[drev::GbL + e];
                    }
                    rf += 5;
                    continue;
                }
                for (int r = 0; r < rows; ++r) {
                    double* row = Md + (rf + r) * md;
                    if (r < 3) {
                        row[ft + r] += 1.;
                        Md[(ft + r) * md + rf + r] += 1.;
                    } else {
                        for (int j = 0; j < 3; ++j) {
                            row[ft + 3 + j] += cr[conrec::Brot + (r - 3) * 3 + j];
                            Md[(ft + 3 + j) * md + rf + r] += cr[conrec::AX + j * 3 + (r - 3)];
                        }
                    }
                    b[rf + r] += cr[conrec::Phi + r];
                }
                for (int e = 0; e < (rows == 3 ? 3 : 6); ++e) b[ft + e] += cr[conrec::Gl + e];
                if (bn >= 0) {  // joint base blocks: B_b = [-I, Btr; 0, Brr], G_b = [-I, tilde; 0, -AX]
                    const int fb = fmap[bn];
                    const double* r1x0 = cr + conrec::R1X0;
                    for (int r = 0; r < rows; ++r) {
                        double* row = Md + (rf + r) * md;
                        if (r < 3) {
                            row[fb + r] -= 1.;
                            Md[(fb + r) * md + rf + r] -= 1.;
                            for (int j = 0; j < 3; ++j) {
                                row[fb + 3 + j] += cr[conrec::Btr + r * 3 + j];
                                Md[(fb + 3 + j) * md + rf + r] += tilde_e(r1x0, r, j);
                            }
                        } else {
                            for (int j = 0; j < 3; ++j) {
                                row[fb + 3 + j] += cr[conrec::Brr + (r - 3) * 3 + j];
                                Md[(fb + 3 + j) * md + rf + r] -= cr[conrec::AX + (r - 3) * 3 + j];
                            }
                        }
                    }
                    double gb[6] = {0., 0., 0., 0., 0., 0.};
                    double lam6[6] = {0., 0., 0., 0., 0., 0.};
                    for (int k = 0; k < rows; ++k) lam6[k] = cr[conrec::lam + k];
                    if (rows == 3) {
                        for (int i = 0; i < 3; ++i) {
                            gb[i] = -lam6[i];
                            for (int k = 0; k < 3; ++k) gb[3 + i] += tilde_e(r1x0, k, i) * lam6[k];
                        }
                    } else {
                        joint_base_transpose_add(cr, lam6, gb);
                    }
                    for (int e = 0; e < 6; ++e) b[fb + e] += gb[e];
                }
                rf += rows;
            }
        }
        __syncthreads();
        // b = -(cond (R - f) on the system rows, Phi on the constraint rows)
        for (int n = tid; n < N; n += NT)  // position-only nodes: components 0..2
            if (fmap[n] >= 0)
                for (int c = 0; c < act[n]; ++c) b[fmap[n] + c] += resid[n * 6 + c] - slab[L.f + n * 6 + c];
        __syncthreads();
        for (int k = tid; k < md; k += NT) b[k] = -(k < nsys ? b[k] * cond : b[k]) + (cnd ? bc[k] : 0.);
        __syncthreads();
        mark(kPhaseConstraints);
        // LU with partial pivoting, in place (the oracle's dense solve)
        for (int k = 0; k < md; ++k) {
            if (warp == 0) {
                double best = -1.;
                int p = k;
                for (int i = k + lane; i < md; i += 32) {
                    const double v = fabs(Md[i * md + k]);
                    if (v > best) {
                        best = v;
                        p = i;
                    }
                }
                for (int o = 16; o > 0; o >>= 1) {
                    const double ob = __shfl_xor_sync(0xffffffffu, best, o);
                    const int op = __shfl_xor_sync(0xffffffffu, p, o);
                    if (ob > best || (ob == best && op < p)) {
                        best = ob;
                        p = op;
                    }
                }
                if (lane == 0) {
                    s_piv = p;
                    if (!(best > 0.)) s_flag |= 2;
                }
            }
            __syncthreads();
            const int p = s_piv;
            if (p != k) {
                for (int j = tid; j < md; j += NT) {
                    const double t0 = Md[k * md + j];
                    Md[k * md + j] = Md[p * md + j];
                    Md[p * md + j] = t0;
                }
                if (tid == 0) {
                    const double t0 = b[k];
                    b[k] = b[p];
                    b[p] = t0;
                }
            }
            __syncthreads();
            // rows below the pivot over the warps, their columns over the lanes;
            // each row's warp forms its multiplier (times the pivot's reciprocal),
            // updates the row and the right-hand side, then stores the multiplier
            // (no other warp reads it)
            const double rd = 1. / Md[k * md + k];
            for (int i = k + 1 + warp; i < md; i += NW) {
                const double l = Md[i * md + k] * rd;
                for (int j = k + 1 + lane; j < md; j += 32) Md[i * md + j] -= l * Md[k * md + j];
                __syncwarp();
                if (lane == 0) {
                    Md[i * md + k] = l;
                    b[i] -= l * b[k];
                }
            }
            __syncthreads();
        }
        mark(kPhaseFactor);
        if (warp == 0) {  // back substitution
            for (int i = md - 1; i >= 0; --i) {
                double s2 = 0.;
                for (int j = i + 1 + lane; j < md; j += 32) s2 += Md[i * md + j] * x[j];
                for (int o = 16; o > 0; o >>= 1) s2 += __shfl_xor_sync(0xffffffffu, s2, o);
                if (lane == 0) x[i] = (b[i] - s2) / Md[i * md + i];
                __syncwarp();
            }
        }
        __syncthreads();
        // multipliers unconditioned; convergence error (calculate_convergence_error.hpp)
        for (int k = nsys + tid; k < md; k += NT) x[k] /= cond;
        __syncthreads();
        if (cnd) cond_back_substitute<NT>(KB, S, smem_raw, fmap, imap, x, xi);
        mark(kPhaseSubstitute);
        // correction of component c of node n
        auto delta_of = [&](int n, int c) { return fmap[n] >= 0 ? x[fmap[n] + c] : xi[imap[n] + c]; };
        double part = 0.;
        for (int n = tid; n < N; n += NT)
            for (int c = 0; c < act[n]; ++c) {
                const double e = delta_of(n, c) / (P.atol + P.rtol * fabs(sqd[n * 6 + c] * h));
                part += e * e;
            }
        if (tid < nc) {
            const double* cr = con + tid * kConStride;
            int rf = nsys;
            for (int c = 0; c < tid; ++c) rf += constraint_rows(KB.con_type[c]);
            const int rows = constraint_rows(KB.con_type[tid]);
            for (int r = 0; r < rows; ++r) {
                const double e = x[rf + r] / (P.atol + P.rtol * fabs(cr[conrec::lam + r]));
                part += e * e;
            }
        }
        for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
        if (lane == 0) red[warp] = part;
        __syncthreads();
        double total = 0.;
        for (int w2 = 0; w2 < NW; ++w2) total += red[w2];
        const double err = sqrt(total / static_cast<double>(nd));
        if (tid == 0 && iter < kMaxNewtonIters) KB.conv[iter] = err;
        iters = iter + 1;
        // update (update_state_prediction.hpp, update_lambda_prediction.hpp)
        for (int n = tid; n < N; n += NT)
            for (int c = 0; c < act[n]; ++c) {
                const double delta = delta_of(n, c);
                sqd[n * 6 + c] += delta / h;
                if (P.dynamic) {
                    sv[n * 6 + c] += P.gamma_prime * delta;
                    svd[n * 6 + c] += P.beta_prime * delta;
                }
            }
        if (tid < nc) {
            double* cr = con + tid * kConStride;
            int rf = nsys;
            for (int c = 0; c < tid; ++c) rf += constraint_rows(KB.con_type[c]);
            const int rows = constraint_rows(KB.con_type[tid]);
            for (int r = 0; r < rows; ++r) cr[conrec::lam + r] += x[rf + r];
        }
        __syncthreads();
        displacement();
        __syncthreads();
        mark(kPhaseUpdate);
        if (s_flag != 0) {
            status = KYN_ERR_SINGULAR;
            break;
        }
        if (!(err == err) || isinf(err)) {
            status = KYN_ERR_NONFINITE;
            break;
        }
        if (err <= 1.) {
            status = KYN_OK;
            break;
        }
    }
    if (s_flag != 0 && status == KYN_NOT_CONVERGED) status = KYN_ERR_INVALID;
    // post-step (step.hpp:86-121) and the resident state
    if (status == KYN_OK) {
        const double fac = (1. - P.alpha_f) / (1. - P.alpha_m);
        for (int k = tid; k < N * 6; k += NT) sa[k] += fac * svd[k];
    }
    __syncthreads();
    for (int k = tid; k < N * 7; k += NT) {
        slab[L.q + k] = sq[k];
        slab[L.q_prev + k] = sqp[k];
    }
    for (int k = tid; k < N * 6; k += NT) {
        slab[L.v + k] = sv[k];
        slab[L.vd + k] = svd[k];
        slab[L.a + k] = sa[k];
        slab[L.q_delta + k] = sqd[k];
    }
    if (status == KYN_OK)
        for (int n = tid; n < N; n += NT) {
            const double* x0 = slab + L.x0 + n * 7;
            for (int c = 0; c < 3; ++c) slab[L.x + n * 7 + c] = x0[c] + sq[n * 7 + c];
            double r[4];
            quat_compose(sq + n * 7 + 3, x0 + 3, r);
            for (int c = 0; c < 4; ++c) slab[L.x + n * 7 + 3 + c] = r[c];
        }
    for (int k = tid; k < N * 9; k += NT) slab[L.tangent + k] = sT[k];
    if (tid < 6 * nc) slab[L.lambda + tid] = con[(tid / 6) * kConStride + conrec::lam + tid % 6];
    if (tid == 0) {
        status_out[KB.plan_model] = status;
        iters_out[KB.plan_model] = iters;
        if (timing)
            for (int k = 0; k < kNumPhases; ++k) atomicAdd(KB.prof + k, s_ph[k]);
    }
    (void)record;  // dense models keep no system dump (kyn_get_system refuses them)
}

// One CTA per dense model.
template <int NT>
__global__ void __launch_bounds__(NT) dense_kernel(const KBeam* __restrict__ beams, StepCoeffs P, int record,
                                                   int* __restrict__ status_out, int* __restrict__ iters_out) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    dense_model_step<NT>(beams[blockIdx.x], P, record, status_out, iters_out, smem_raw);
}

// ---- the kernel ------------------------------------------------------------------
// Resident CTAs per SM that each instance is compiled for (its register budget
// is 65536 / (NT * this), 128 registers per thread for all three).  Three
// 256-thread CTAs per SM in the FP32 form (80 registers) would fit its shared
// memory up to 16 nodes, but the spills land in the pivot loops and cost more
// than the third beam per SM hides.
__host__ __device__ constexpr int step_min_blocks(int real_bytes, int nt) {
    return (void)real_bytes, nt == 128 ? 4 : nt == 256 ? 2 : 1;
}

// LUMP: the instance that also adds point masses and springs (KBeam::lumped);
// beams without them run the instance compiled without that code, whose
// registers it would otherwise crowd.
// GJ: the instance that also carries the register Gauss-Jordan solve
// (KYN_SOLVER_GAUSS_JORDAN); the default instances carry only the panel LU,
// whose register allocation the Gauss-Jordan tile would otherwise crowd.
template <typename TR, int NT, bool LUMP, bool GJ = false>
__global__ void __launch_bounds__(NT, step_min_blocks(sizeof(TR), NT))
    step_kernel(const KBeam* __restrict__ beams, StepCoeffs P, int record,
                int* __restrict__ status_out, int* __restrict__ iters_out) {
    static_assert(NT == 128 || NT == 256 || NT == 512, "step kernel runs with 128, 256 or 512 threads");
    constexpr int NW = NT / 32;  // warps
    constexpr int NG = NT / 16;  // quadrature-point groups of 16 threads
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const KBeam& KB = beams[blockIdx.x];
    const int N = KB.N, Q = KB.Q, nc = KB.nc;
    const int n6 = 6 * N;
    const int m = 6 * (N - nc);   // free-node block size
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int chain = KB.hub;  // hub chain length (0: no hub)
    const bool hub = chain != 0;
    const bool drive = LUMP && chain > 1;  // drive trains run in the LUMP instance only
    if (!LUMP && chain > 1) {  // launch-plan error: refuse rather than solve without the chain
        if (tid == 0 && KB.rank == 0) {
            status_out[KB.plan_model] = KYN_ERR_UNSUPPORTED;
            iters_out[KB.plan_model] = 0;
        }
        return;
    }
    const Smem S = make_smem(N, Q, nc, sizeof(TR), NT, drive ? 2 : (hub ? 1 : 0));
    const SlabLayout L = make_slab_layout(N, Q);
    double* __restrict__ slab = KB.slab;

    TR* A = reinterpret_cast<TR*>(smem_raw + S.A);
    const int ldA = S.ldA;
    using TG = TR;  // element type of G: FP64 form double, FP32 form float
    TG* G = reinterpret_cast<TG*>(smem_raw + S.G);
    double* Fc = reinterpret_cast<double*>(smem_raw + S.Fc);
    double* Fdig = reinterpret_cast<double*>(smem_raw + S.Fdig);
    double* phi = reinterpret_cast<double*>(smem_raw + S.phi);
    double* dphi = reinterpret_cast<double*>(smem_raw + S.dphi);
    double* dphiJ = reinterpret_cast<double*>(smem_raw + S.dphiJ);
    double* qpw = reinterpret_cast<double*>(smem_raw + S.qpw);
    double* sq = reinterpret_cast<double*>(smem_raw + S.q);
    double* sqp = reinterpret_cast<double*>(smem_raw + S.q_prev);
    double* sv = reinterpret_cast<double*>(smem_raw + S.v);
    double* svd = reinterpret_cast<double*>(smem_raw + S.vd);
    double* sa = reinterpret_cast<double*>(smem_raw + S.a);
    double* sqd = reinterpret_cast<double*>(smem_raw + S.qd);
    double* sT = reinterpret_cast<double*>(smem_raw + S.T);
    double* hb = hub ? reinterpret_cast<double*>(smem_raw + S.hub) : nullptr;  // hub record
    // drive train: chain records 1 (revolute target) and 2 (optional), and the
    // record the beam roots join (the last of the chain)
    double* hA = drive ? hb + hubsm::n1 : nullptr;
    double* hH = (drive && chain == 3) ? hb + hubsm::n2 : nullptr;
    double* hj = drive ? (hH ? hH : hA) : hb;
    double* resid = reinterpret_cast<double*>(smem_raw + S.resid);
    double* bp = reinterpret_cast<double*>(smem_raw + S.b);
    double* xs = reinterpret_cast<double*>(smem_raw + S.xs);
    double* rpiv = reinterpret_cast<double*>(smem_raw + S.rpiv);
    double* stage = reinterpret_cast<double*>(smem_raw + S.stage);
    double* con = reinterpret_cast<double*>(smem_raw + S.con);
    double* gscr = reinterpret_cast<double*>(smem_raw + S.A);  // quadrature phase only
    double* red = reinterpret_cast<double*>(smem_raw + S.red);
    int* pos = reinterpret_cast<int*>(smem_raw + S.pos);
    __shared__ int s_flag;
    __shared__ unsigned long long s_ph[kNumPhases];
    // sections of the next quadrature phase: one bulk copy per Newton
    // iteration (slab from x0' on -> the A region after the group scratch)
    uint64_t* sec_bar = reinterpret_cast<uint64_t*>(smem_raw + S.bar);
    double* sec = reinterpret_cast<double*>(smem_raw + S.sec);
    const uint32_t sec_bytes = static_cast<uint32_t>(sec_doubles(Q)) * 8u;
    uint32_t sec_issued = 0, sec_waited = 0;  // copies issued / completed (thread 0 issues)
    const bool bulk = P.bulk_sections != 0;
    auto sec_prefetch = [&]() {  // all threads, once every use of the region has ended
        if (!bulk) return;
        proxy_fence_async_smem();
        __syncthreads();
        if (tid == 0) bulk_copy_g2s(sec, slab + L.x0p, sec_bytes, sec_bar);
        ++sec_issued;
    };
    auto sec_wait = [&]() {  // all threads
        if (!bulk) return;
        if (!mbar_wait(sec_bar, sec_waited & 1u) && tid == 0) atomicOr(&s_flag, 8);
        ++sec_waited;
    };

    const double h = P.h;
    // Optional phase timing: thread 0 reads the SM clock at phase boundaries
    // (after a CTA barrier) and adds the cycles to prof[phase] at the end.
    const bool timing = KB.prof != nullptr;
    long long ph_t = 0;
    if (timing && tid == 0) {
        for (int k = 0; k < kNumPhases; ++k) s_ph[k] = 0ull;
        ph_t = clock64();
    }
    auto mark = [&](int phase) {
        if (timing && tid == 0) {
            const long long t = clock64();
            s_ph[phase] += static_cast<unsigned long long>(t - ph_t);
            ph_t = t;
        }
    };

    // ---- load constants and state ------------------------------------------
    for (int k = tid; k < Q * N; k += NT) {
        phi[k] = slab[L.phi + k];
        dphi[k] = slab[L.dphi + k];
        dphiJ[k] = slab[L.dphiJ + k];
    }
    for (int k = tid; k < Q * 4; k += NT) qpw[k] = slab[L.qpw + k];

    for (int k = tid; k < N * 7; k += NT) sq[k] = slab[L.q + k];
    for (int k = tid; k < N * 6; k += NT) {
        sv[k] = slab[L.v + k];
        svd[k] = slab[L.vd + k];
        sa[k] = slab[L.a + k];
    }
    if (tid < nc) {
        double* c = con + tid * kConStride;
        for (int k = 0; k < 7; ++k) c[conrec::inp + k] = slab[L.con_input + tid * 7 + k];
        for (int k = 0; k < 6; ++k) c[conrec::lam + k] = 0.;  // ResetConstraints
    }
    if (hub) {
        for (int k = tid; k < kHubDoubles; k += NT) hb[k] = slab[L.hub + k];
        if (tid == 0) {
            double* br = hb + hubsm::bc;
            for (int k = 0; k < 7; ++k) br[conrec::inp + k] = slab[L.hub + hubrec::input + k];
            for (int k = 0; k < 6; ++k) br[conrec::lam + k] = 0.;  // ResetConstraints
        }
    }
    if (drive) {
        for (int k = tid; k < (chain - 1) * kHubDoubles; k += NT)
            hb[hubsm::n1 + (k / kHubDoubles) * (hubsm::n2 - hubsm::n1) + k % kHubDoubles] =
                slab[L.hub + kHubDoubles + k];
        if (tid == 0)
            for (int k = 0; k < 6; ++k) {  // ResetConstraints
                hb[hubsm::rev + revrec::lam + k] = 0.;
                hb[hubsm::ah + conrec::lam + k] = 0.;
            }
    }
    if (tid == 0) {
        // Free nodes first, constrained nodes last (in constraint order).
        int p = 0;
        for (int n = 0; n < N; ++n) {
            bool constrained = false;
            for (int c = 0; c < nc; ++c) constrained |= (KB.con_node[c] == n);
            if (!constrained) pos[n] = p++;
        }
        for (int c = 0; c < nc; ++c) pos[KB.con_node[c]] = p++;
        s_flag = 0;
        mbar_init(sec_bar);
    }
    __syncthreads();
    sec_prefetch();

    if (sizeof(TR) == 4 && (Q & 1))  // zero pad point of the FP32 integration GEMM
        for (int k = tid; k < 4 * 56; k += NT) G[4 * Q * 56 + k] = TG(0);

    // ---- PredictNextState (src/step/predict_next_state.hpp:14-47) ------------
    for (int k = tid; k < N * 7; k += NT) sqp[k] = sq[k];
    for (int k = tid; k < N * 6; k += NT) {
        const double v_p = sv[k], vd_p = svd[k], a_p = sa[k];
        svd[k] = 0.;
        const double an = (P.alpha_f * vd_p - P.alpha_m * a_p) / (1. - P.alpha_m);
        sa[k] = an;
        sv[k] = v_p + h * (1. - P.gamma) * a_p + P.gamma * h * an;
        sqd[k] = v_p + (0.5 - P.beta) * h * a_p + P.beta * h * an;
    }
    // hub-chain records: thread NT-1-r owns record r (evaluated where used, so
    // that the instances without a drive train keep no extra register live)
    auto chain_rec = [&]() -> double* {
        return tid == NT - 1 ? hb : (tid == NT - 2) ? hA : (tid == NT - 3) ? hH : nullptr;
    };
    if (hub && chain_rec()) {  // the hub node(s): same predictor
        double* r = chain_rec();
        for (int k = 0; k < 7; ++k) r[hubrec::q_prev + k] = r[hubrec::q + k];
        for (int k = 0; k < 6; ++k) {
            const double v_p = r[hubrec::v + k], vd_p = r[hubrec::vd + k], a_p = r[hubrec::a + k];
            r[hubrec::vd + k] = 0.;
            const double an = (P.alpha_f * vd_p - P.alpha_m * a_p) / (1. - P.alpha_m);
            r[hubrec::a + k] = an;
            r[hubrec::v + k] = v_p + h * (1. - P.gamma) * a_p + P.gamma * h * an;
            r[hubrec::q_delta + k] = v_p + (0.5 - P.beta) * h * a_p + P.beta * h * an;
        }
    }
    __syncthreads();
    // CalculateDisplacement (src/state/calculate_displacement.hpp:25-50)
    auto displacement = [&]() {
        for (int n = tid; n < N; n += NT) {
            for (int c = 0; c < 3; ++c) sq[n * 7 + c] = sqp[n * 7 + c] + h * sqd[n * 6 + c];
            const double d[3] = {h * sqd[n * 6 + 3], h * sqd[n * 6 + 4], h * sqd[n * 6 + 5]};
            double qd4[4], qn[4];
            rotvec_to_quat(d, qd4);
            quat_compose(qd4, sqp + n * 7 + 3, qn);
            for (int c = 0; c < 4; ++c) sq[n * 7 + 3 + c] = qn[c];
        }
        if (hub && chain_rec()) {
            double* hq = chain_rec() + hubrec::q;
            const double* hqp = chain_rec() + hubrec::q_prev;
            const double* hqd = chain_rec() + hubrec::q_delta;
            for (int c = 0; c < 3; ++c) hq[c] = hqp[c] + h * hqd[c];
            const double d[3] = {h * hqd[3], h * hqd[4], h * hqd[5]};
            double qd4[4], qn[4];
            rotvec_to_quat(d, qd4);
            quat_compose(qd4, hqp + 3, qn);
            for (int c = 0; c < 4; ++c) hq[3 + c] = qn[c];
        }
    };
    displacement();
    __syncthreads();
    mark(kPhaseLoadPredict);

    int status = KYN_NOT_CONVERGED;
    int iters = 0;
    const cg::cluster_group cluster = cg::this_cluster();
    const bool clustered = KB.model_beams > 1;

    int extra = 0;  // refinement corrections taken after convergence (FP32 form)
    for (int iter = 0; iter < P.max_iter + extra; ++iter) {
        // ---- tangent operator (src/system/calculate_tangent_operator.hpp:26-65)
        // Only the rotational 3x3 block of the stored (transposed) operator is kept.
        auto tangent_op = [&](const double* qd, double* T) {
            const double rv[3] = {h * qd[3], h * qd[4], h * qd[5]};
            const double ph = sqrt(rv[0] * rv[0] + rv[1] * rv[1] + rv[2] * rv[2]);
            double sn, cs;
            sincos(ph, &sn, &cs);
            const double t1 = (ph > 1.e-16) ? (cs - 1.) / (ph * ph) : 0.;
            const double t2 = (ph > 1.e-16) ? (1. - sn / ph) / (ph * ph) : 0.;
            for (int i = 0; i < 3; ++i) {
                for (int j = 0; j < 3; ++j) {
                    // m1 = t2*(rv~ rv~) + t1*rv~ ; T_rot = I + m1 ; stored transposed
                    double rr = 0.;
                    for (int k = 0; k < 3; ++k) rr += tilde_e(rv, j, k) * tilde_e(rv, k, i);
                    T[i * 3 + j] = (i == j ? 1. : 0.) + (t1 * tilde_e(rv, j, i) + t2 * rr);
                }
            }
        };
        for (int n = tid; n < N; n += NT) tangent_op(sqd + n * 6, sT + n * 9);
        if (hub && chain_rec()) tangent_op(chain_rec() + hubrec::q_delta, chain_rec() + hubrec::tangent);

        // ---- quadrature-point values (calculate_quadrature_point_values.hpp) ---
        sec_wait();
        qp_phase<TG, NT>(N, Q, phi, dphiJ, qpw, sq, sv, svd, slab, L, KB.gravity, P.beta_prime,
                         P.gamma_prime, gscr, G, Fc, Fdig, bulk ? sec : nullptr);
        __syncthreads();
        mark(kPhaseQuadrature);

        // ---- residual integration (integrate_residual_vector.hpp:33-50) ----------
        for (int t = tid; t < N * 6; t += NT) {
            const int n = t / 6, c = t % 6;
            double acc = 0.;
            for (int qp = 0; qp < Q; ++qp) {
                const double w = qpw[qp * 4], wJ = qpw[qp * 4 + 2];
                acc += (w * dphi[qp * N + n]) * Fc[qp * 6 + c] +
                       (wJ * phi[qp * N + n]) * Fdig[qp * 6 + c];
            }
            resid[t] = acc - slab[L.fx + t];
        }

        // ---- stiffness + inertia integration and S T + I (integrate_*_matrix.hpp,
        //      calculate_system_matrix.hpp), scaled by the conditioner into A.
        //      For node pair (i,j):  C_ij = sum_q sum_m coef_m(i,j,q) G[4q+m]  with
        //      coef = (phi_i phi_j, phi_i phi'_j, phi'_i phi'_j, phi'_i phi_j) and G the
        //      weighted blocks written by the quadrature phase (K/inertia, P, C, O
        //      terms).  C_ij holds [S+I left | S right | I right]; then
        //      SM_ij = [C_L | C_RS T_j + C_RI] (T_j is identity on the translational
        //      block).  The pair GEMM runs on the FP64 tensor cores: each warp owns
        //      tiles of 8 pairs and all 7 column tiles, one k-step of 4 (m = 0..3) per
        //      point, and writes SM_ij from its accumulators (column layout: gcol).
        __syncthreads();
        {
            const int P2 = N * N;
            const int s4 = lane & 3;
            const double* fi_tab = (s4 < 2) ? phi : dphi;
            const double* fj_tab = (s4 == 0 || s4 == 3) ? phi : dphi;
            const double cond = P.conditioner;
            if constexpr (sizeof(TR) == 8) {
                // FP64 tensor cores, m8n8k4: 8 pairs per tile, one point per k-step
                for (int p0 = 8 * warp; p0 < P2; p0 += 8 * NW) {
                    const int prow = p0 + (lane >> 2);
                    const bool valid = prow < P2;
                    const int i = valid ? prow / N : 0, jn = valid ? prow % N : 0;
                    double acc[7][2];
#pragma unroll
                    for (int nt = 0; nt < 7; ++nt) acc[nt][0] = acc[nt][1] = 0.;
                    for (int q = 0; q < Q; ++q) {
                        const double av = valid ? fi_tab[q * N + i] * fj_tab[q * N + jn] : 0.;
                        const TG* gq = G + (4 * q + s4) * 56 + (lane >> 2);
#pragma unroll
                        for (int nt = 0; nt < 7; ++nt) dmma884(acc[nt][0], acc[nt][1], av, gq[nt * 8]);
                    }
                    if (valid)
                        store_pair_block(A, ldA, pos, sT, i, jn, s4, cond,
                                         [&](int t) { return acc[t >> 1][t & 1]; });
                }
            } else {
                // FP32 form: TF32 tensor cores with the 3-term split (hi*hi + hi*lo +
                // lo*hi, FP32 accumulation), m16n8k8: 16 pairs per tile, two points
                // per k-step (an odd Q reads the zero pad point).
                const int g8 = lane >> 2;
                const int QK = (Q + 1) >> 1;
                for (int p0 = 16 * warp; p0 < P2; p0 += 16 * NW) {
                    const int pa = p0 + g8, pb = p0 + g8 + 8;
                    const bool va = pa < P2, vb = pb < P2;
                    const int ia = va ? pa / N : 0, ja = va ? pa % N : 0;
                    const int ib = vb ? pb / N : 0, jb = vb ? pb % N : 0;
                    float acc[7][4];
#pragma unroll
                    for (int nt = 0; nt < 7; ++nt) acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.f;
                    for (int ks = 0; ks < QK; ++ks) {
                        const int q0 = 2 * ks, q1 = 2 * ks + 1;
                        const bool q1ok = q1 < Q;
                        const int q1c = q1ok ? q1 : q0;
                        float av[4];
                        av[0] = va ? static_cast<float>(fi_tab[q0 * N + ia] * fj_tab[q0 * N + ja]) : 0.f;
                        av[1] = vb ? static_cast<float>(fi_tab[q0 * N + ib] * fj_tab[q0 * N + jb]) : 0.f;
                        av[2] = (va && q1ok) ? static_cast<float>(fi_tab[q1c * N + ia] * fj_tab[q1c * N + ja]) : 0.f;
                        av[3] = (vb && q1ok) ? static_cast<float>(fi_tab[q1c * N + ib] * fj_tab[q1c * N + jb]) : 0.f;
                        unsigned ah[4], al[4];
#pragma unroll
                        for (int r = 0; r < 4; ++r) split_tf32(av[r], ah[r], al[r]);
                        const TG* g0 = G + (4 * q0 + s4) * 56 + g8;
                        const TG* g1 = G + (4 * q1 + s4) * 56 + g8;
#pragma unroll
                        for (int nt = 0; nt < 7; ++nt) {
                            unsigned bh[2], bl[2];
                            split_tf32(static_cast<float>(g0[nt * 8]), bh[0], bl[0]);
                            split_tf32(static_cast<float>(g1[nt * 8]), bh[1], bl[1]);
                            mma_tf32(acc[nt], al, bh);
                            mma_tf32(acc[nt], ah, bl);
                            mma_tf32(acc[nt], ah, bh);
                        }
                    }
                    if (va)
                        store_pair_block(A, ldA, pos, sT, ia, ja, s4, cond,
                                         [&](int t) { return static_cast<double>(acc[t >> 1][t & 1]); });
                    if (vb)
                        store_pair_block(A, ldA, pos, sT, ib, jb, s4, cond,
                                         [&](int t) { return static_cast<double>(acc[t >> 1][2 + (t & 1)]); });
                }
            }
        }
        __syncthreads();
        if (LUMP && KB.n_mass + KB.n_spring > 0) {  // point masses and springs at this CTA's nodes
            for (int n = tid; n < N; n += NT)
                add_lumped_terms(n, KB.lumped, KB.n_mass, KB.n_spring, sq, sv, svd, sT, KB.gravity,
                                 P.beta_prime, P.gamma_prime, P.conditioner, pos, A, ldA, resid);
            __syncthreads();
        }
        mark(kPhaseIntegrate);

        // ---- constraints (calculate_constraint_residual_gradient.hpp:60-320) -------
        if (warp == NW - 1 && lane < nc) {
            const int tn = KB.con_node[lane];
            constraint_record(con + lane * kConStride, KB.con_type[lane], sq + tn * 7, KB.con_X0[lane],
                              sT + tn * 9, hub ? hj + hubrec::q : nullptr,
                              hub ? hj + hubrec::tangent : nullptr, KB.con_axis[lane]);
        }
        if (hub && warp == NW - 1 && lane == nc)  // the hub's own boundary condition
            constraint_record(hb + hubsm::bc, KB.hub_con_type, hb + hubrec::q, hb + hubrec::X0,
                              hb + hubrec::tangent, nullptr, nullptr, nullptr);
        if (drive && warp == NW - 1 && lane == nc + 1)  // revolute joint record 0 -> 1
            revolute_record(hb + hubsm::rev, hb, hA);
        if (drive && hH && warp == NW - 1 && lane == nc + 2)  // rigid joint record 1 -> 2
            constraint_record(hb + hubsm::ah, KYN_CONSTRAINT_RIGID_JOINT, hH + hubrec::q, hH + hubrec::X0,
                              hH + hubrec::tangent, hA + hubrec::q, hA + hubrec::tangent, nullptr);
        __syncthreads();

        // ---- right-hand side: b = -cond (-f + R + G^T lambda) (assemble_system_residual.hpp,
        //      solve_system.hpp:20-24) in permuted order --------------------------------
        for (int t = tid; t < n6; t += NT) {
            const int n = t / 6, c = t % 6;
            double val = -slab[L.f + t] + resid[t];
            for (int k = 0; k < nc; ++k)
                if (KB.con_node[k] == n) val += con[k * kConStride + conrec::Gl + c];
            bp[6 * pos[n] + c] = -(val * P.conditioner);
        }
        if (record && KB.dump) {
            // Dump of the assembled local system (natural node order, then constraints):
            // matrix [nl][nl], then rhs [nl], then solution [nl]; nl = n6 + 6 nc.
            const int nl = n6 + 6 * nc;
            double* D = KB.dump;
            for (int t = tid; t < nl * nl; t += NT) D[t] = 0.;
        }
        __syncthreads();
        if (record && KB.dump) {
            const int nl = n6 + 6 * nc;
            double* D = KB.dump;
            for (int t = tid; t < n6 * n6; t += NT) {
                const int r = t / n6, c = t % n6;
                D[r * nl + c] = static_cast<double>(A[(6 * pos[r / 6] + r % 6) * ldA + 6 * pos[c / 6] + c % 6]);
            }
            for (int t = tid; t < n6; t += NT) D[nl * nl + t] = bp[6 * pos[t / 6] + t % 6];
            if (tid < nc) {
                const double* cr = con + tid * kConStride;
                const int tn = KB.con_node[tid];
                const int r0 = n6 + 6 * tid;
                for (int k = 0; k < 3; ++k) {
                    D[(r0 + k) * nl + 6 * tn + k] = 1.;            // B translational block
                    D[(6 * tn + k) * nl + r0 + k] = 1.;            // grad^T translational block
                }
                for (int i = 0; i < 3; ++i)
                    for (int j = 0; j < 3; ++j) {
                        D[(r0 + 3 + i) * nl + 6 * tn + 3 + j] = cr[conrec::Brot + i * 3 + j];
                        D[(6 * tn + 3 + i) * nl + r0 + 3 + j] = cr[conrec::AX + i * 3 + j];
                    }
                for (int k = 0; k < 6; ++k) D[nl * nl + r0 + k] = -cr[conrec::Phi + k];
            }
        }

        __syncthreads();
        mark(kPhaseConstraints);

        // ---- solve -----------------------------------------------------------------
        // (S1) constrained node corrections: B x_r = -Phi.  With a hub, its
        //      correction comes first (its BC rows), then each rigid joint gives
        //      the root correction: B_t x_root = -Phi - B_base x_hub.
        if (hub) {
            if (tid == 0) {
                const double* br = hb + hubsm::bc;
                double* xh = hb + hubsm::xh;
                for (int k = 0; k < 3; ++k) xh[k] = -br[conrec::Phi + k];
                const double rhs[3] = {-br[conrec::Phi + 3], -br[conrec::Phi + 4], -br[conrec::Phi + 5]};
                double y[3] = {0., 0., 0.};
                if (!solve3(br + conrec::Brot, rhs, y)) atomicOr(&s_flag, 2);
                for (int k = 0; k < 3; ++k) xh[3 + k] = y[k];
                if (drive) {
                    // Drive train: the revolute rows fix record 1's translation and
                    // two of its rotation components; the third, the shaft rotation
                    // theta, stays free.  x_1 = cA + theta nA, nA spanning the null
                    // space of B_t; the chain's later corrections are affine in
                    // theta as well (cH + theta dH).  Test vectors w (G w = 0 with
                    // the gradients G, not G T) project the equilibrium rows onto
                    // the free rotation: w_1 = [0, joint axis].
                    const double* rv = hb + hubsm::rev;
                    double* cA = hb + hubsm::cA;
                    double* nA = hb + hubsm::nA;
                    double* wA = hb + hubsm::wA;
                    for (int k = 0; k < 3; ++k) {
                        cA[k] = -rv[revrec::Phi + k] + xh[k];
                        nA[k] = 0.;
                        wA[k] = 0.;
                        wA[3 + k] = rv[revrec::x + k];
                    }
                    const double* b0 = rv + revrec::Bt;
                    const double* b1 = rv + revrec::Bt + 3;
                    double r2[2];
                    for (int i = 0; i < 2; ++i) {
                        r2[i] = -rv[revrec::Phi + 3 + i];
                        for (int k = 0; k < 3; ++k) r2[i] -= rv[revrec::Bb + i * 3 + k] * xh[3 + k];
                    }
                    // minimum-norm particular solution B_t^T (B_t B_t^T)^-1 r2
                    const double g00 = b0[0] * b0[0] + b0[1] * b0[1] + b0[2] * b0[2];
                    const double g01 = b0[0] * b1[0] + b0[1] * b1[1] + b0[2] * b1[2];
                    const double g11 = b1[0] * b1[0] + b1[1] * b1[1] + b1[2] * b1[2];
                    const double det = g00 * g11 - g01 * g01;
                    if (!(fabs(det) > 0.)) atomicOr(&s_flag, 2);
                    const double l0 = (g11 * r2[0] - g01 * r2[1]) / det;
                    const double l1 = (g00 * r2[1] - g01 * r2[0]) / det;
                    for (int k = 0; k < 3; ++k) cA[3 + k] = b0[k] * l0 + b1[k] * l1;
                    nA[3] = b0[1] * b1[2] - b0[2] * b1[1];
                    nA[4] = b0[2] * b1[0] - b0[0] * b1[2];
                    nA[5] = b0[0] * b1[1] - b0[1] * b1[0];
                    if (hH) {
                        const double* ah = hb + hubsm::ah;
                        bool ok = joint_target_correction(ah, cA, 1., hb + hubsm::cH);
                        ok &= joint_target_correction(ah, nA, 0., hb + hubsm::dH);
                        ok &= joint_target_test(ah, wA, hb + hubsm::wH);
                        if (!ok) atomicOr(&s_flag, 2);
                    }
                }
            }
            __syncthreads();
        }
        if (drive && tid < nc) {
            // roots: x_root = c_r + theta d_r from the corrections of the record
            // they join; d_r waits in rpiv's constrained rows (the LU uses rpiv
            // below m only) for the second right-hand side
            double* cr = con + tid * kConStride;
            const int pr = 6 * pos[KB.con_node[tid]];
            double c6[6], d6[6];
            if (is_hub_joint(KB.con_type[tid])) {
                const double* cb = hb + (hH ? hubsm::cH : hubsm::cA);
                const double* db = hb + (hH ? hubsm::dH : hubsm::nA);
                bool ok = joint_target_correction(cr, cb, 1., c6);
                ok &= joint_target_correction(cr, db, 0., d6);
                ok &= joint_target_test(cr, hb + (hH ? hubsm::wH : hubsm::wA), cr + conrec::wr);
                if (!ok) atomicOr(&s_flag, 2);
            } else {
                for (int k = 0; k < 3; ++k) {
                    c6[k] = -cr[conrec::Phi + k];
                    d6[k] = d6[3 + k] = 0.;
                }
                const double rr[3] = {-cr[conrec::Phi + 3], -cr[conrec::Phi + 4], -cr[conrec::Phi + 5]};
                if (!solve3(cr + conrec::Brot, rr, c6 + 3)) atomicOr(&s_flag, 2);
                for (int k = 0; k < 6; ++k) cr[conrec::wr + k] = 0.;
            }
            for (int k = 0; k < 6; ++k) {
                xs[pr + k] = c6[k];
                rpiv[pr + k] = d6[k];
                cr[conrec::dr + k] = d6[k];
            }
        } else if (tid < nc) {
            const double* cr = con + tid * kConStride;
            const int pr = 6 * pos[KB.con_node[tid]];
            double rt[3], rr[3];
            for (int k = 0; k < 3; ++k) {
                rt[k] = -cr[conrec::Phi + k];
                rr[k] = -cr[conrec::Phi + 3 + k];
            }
            if (is_hub_joint(KB.con_type[tid])) {
                const double* xh = hb + hubsm::xh;
                for (int i = 0; i < 3; ++i) {
                    rt[i] += xh[i];
                    for (int k = 0; k < 3; ++k) {
                        rt[i] -= cr[conrec::Btr + i * 3 + k] * xh[3 + k];
                        rr[i] -= cr[conrec::Brr + i * 3 + k] * xh[3 + k];
                    }
                }
            }
            for (int k = 0; k < 3; ++k) xs[pr + k] = rt[k];
            double y[3] = {0., 0., 0.};
            if (!solve3(cr + conrec::Brot, rr, y)) atomicOr(&s_flag, 2);
            for (int k = 0; k < 3; ++k) xs[pr + 3 + k] = y[k];
        }
        __syncthreads();
        // (S2) free-row right-hand side, folded into column m of A (and kept in
        //      FP64 in bp[0:m]); a drive train adds the second right-hand side
        //      -A_fr d_r in column m + 1 (FP64 copy in rhs2)
        double* gjv = reinterpret_cast<double*>(smem_raw + S.G + gj_vec_offset(sizeof(TR), NT));
        double* r64 = gjv;                 // [n6] residual of the linear solve
        double* rhs2 = gjv + n6;           // [n6] second right-hand side (drive train)
        double* x2 = gjv + 2 * n6;         // [n6] its solution
        double* red4 = gjv + 4 * n6;       // [64] reductions of the refinement
        for (int i = tid; i < m; i += NT) {
            double r = bp[i], r2 = 0.;
            for (int j = m; j < n6; ++j) {
                r -= static_cast<double>(A[i * ldA + j]) * xs[j];
                if (drive) r2 -= static_cast<double>(A[i * ldA + j]) * rpiv[j];
            }
            A[i * ldA + m] = static_cast<TR>(r);
            bp[i] = r;
            if (drive) {
                A[i * ldA + m + 1] = static_cast<TR>(r2);
                rhs2[i] = r2;
            }
        }
        __syncthreads();
        mark(kPhaseEliminate);
        // (S3) the free block: Gauss-Jordan in registers where it fits the grid
        //      (FP64 form: solve; FP32 form: inverse, then FP64-residual
        //      refinement), else the panel LU.  x1 -> xs[0:m], x2 -> x2[0:m].
        constexpr bool kInv = sizeof(TR) == 4;
        const int nrhs = drive ? 2 : 1;
        const bool use_gj = GJ && P.solver == KYN_SOLVER_GAUSS_JORDAN && m > 0 && (m & 1) == 0 &&
                            gj_fits<TR, NT>(m, kInv ? m : m + nrhs);
        if (use_gj) {
          if constexpr (GJ) {
            TR R[GJTile<TR, NT>::RT][GJTile<TR, NT>::CT];
            gj_eliminate<TR, NT, kInv>(A, ldA, m, nrhs, reinterpret_cast<TR*>(smem_raw + S.G), &s_flag, R);
            mark(kPhaseFactor);
            // Backward error of a solve: max|b - A x| / (||A|| ||x|| + ||b||),
            // infinity norms, FP64, A as assembled (its FP32 rounding in the
            // FP32 form).  Returns the same value in every thread.
            auto backward_error = [&](const double* x, const double* b, double* res) -> double {
                double ra = 0., xa = 0., ba = 0., aa = 0.;
                constexpr int PR = NT / kGJCols;
                const int ri = tid / kGJCols, cj = tid % kGJCols;
#pragma unroll
                for (int a = 0; a < GJTile<TR, NT>::RT; ++a) {
                    const int i = ri + a * PR;
                    if (a * PR >= m) break;
                    double acc = 0., asum = 0.;
#pragma unroll
                    for (int bb = 0; bb < GJTile<TR, NT>::CT; ++bb) {
                        const int j = cj + bb * kGJCols;
                        if (j < m && i < m) {
                            const double aij = static_cast<double>(A[i * ldA + j]);
                            acc = fma(aij, x[j], acc);
                            asum += fabs(aij);
                            if (a == 0) xa = fmax(xa, fabs(x[j]));
                        }
                    }
#pragma unroll
                    for (int o = 8; o > 0; o >>= 1) {
                        acc += __shfl_xor_sync(0xffffffffu, acc, o);
                        asum += __shfl_xor_sync(0xffffffffu, asum, o);
                    }
                    if (i < m) {
                        const double rv = b[i] - acc;
                        if (cj == 0) res[i] = rv;
                        ra = fmax(ra, fabs(rv));
                        ba = fmax(ba, fabs(b[i]));
                        aa = fmax(aa, asum);
                    }
                }
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    ra = fmax(ra, __shfl_xor_sync(0xffffffffu, ra, o));
                    xa = fmax(xa, __shfl_xor_sync(0xffffffffu, xa, o));
                    ba = fmax(ba, __shfl_xor_sync(0xffffffffu, ba, o));
                    aa = fmax(aa, __shfl_xor_sync(0xffffffffu, aa, o));
                }
                if (lane == 0) {
                    red4[4 * warp] = ra;
                    red4[4 * warp + 1] = xa;
                    red4[4 * warp + 2] = ba;
                    red4[4 * warp + 3] = aa;
                }
                __syncthreads();
                ra = xa = ba = aa = 0.;
                for (int w2 = 0; w2 < NW; ++w2) {
                    ra = fmax(ra, red4[4 * w2]);
                    xa = fmax(xa, red4[4 * w2 + 1]);
                    ba = fmax(ba, red4[4 * w2 + 2]);
                    aa = fmax(aa, red4[4 * w2 + 3]);
                }
                __syncthreads();  // red4 is reused by the next call
                const double den = aa * xa + ba;
                return den > 0. ? ra / den : 0.;
            };
            if constexpr (!kInv) {
                gj_extract<TR, NT>(R, m, m, xs);
                if (drive) gj_extract<TR, NT>(R, m, m + 1, x2);
                __syncthreads();
                // guard of the unpivoted elimination: the backward error of the
                // solve, counted (checked, above kGJBackwardErrorMax, largest)
                for (int rhs = 0; rhs < nrhs; ++rhs) {
                    const double eta = backward_error(rhs ? x2 : xs, rhs ? rhs2 : bp, r64);
                    if (tid == 0 && P.diag) {
                        atomicAdd(P.diag + kDiagChecked, 1ull);
                        if (!(eta <= kGJBackwardErrorMax)) atomicAdd(P.diag + kDiagGuardTrips, 1ull);
                        if (eta == eta)
                            atomicMax(P.diag + kDiagMaxBackwardError,
                                      static_cast<unsigned long long>(__double_as_longlong(eta)));
                    }
                }
            } else {
                // FP32 inverse in R; x = R b, then sweeps x += R (b - A x) with
                // the residual in FP64 until its backward error is at most
                // refine_tol (or refine_sweeps sweeps)
                for (int rhs = 0; rhs < nrhs; ++rhs) {
                    double* x = rhs ? x2 : xs;
                    const double* b = rhs ? rhs2 : bp;
                    double amax;
                    gj_matvec<TR, NT, true>(R, A, ldA, m, b, nullptr, x, amax);
                    __syncthreads();
                    for (int sweep = 1;; ++sweep) {
                        const double eta = backward_error(x, b, r64);
                        const bool done = eta <= P.refine_tol;
                        if (tid == 0 && P.diag) {
                            if (done || sweep > P.refine_sweeps) {
                                atomicAdd(P.diag + kDiagChecked, 1ull);
                                if (eta == eta)
                                    atomicMax(P.diag + kDiagMaxBackwardError,
                                              static_cast<unsigned long long>(__double_as_longlong(eta)));
                            }
                            if (!done && sweep > P.refine_sweeps) atomicAdd(P.diag + kDiagRefineShort, 1ull);
                            if (!done && sweep <= P.refine_sweeps) atomicAdd(P.diag + kDiagRefineSweeps, 1ull);
                        }
                        if (done || sweep > P.refine_sweeps) break;
                        // x += R r: one row group's 16 threads sum their columns
                        constexpr int PR = NT / kGJCols;
                        const int ri = tid / kGJCols, cj = tid % kGJCols;
#pragma unroll
                        for (int a = 0; a < GJTile<TR, NT>::RT; ++a) {
                            const int i = ri + a * PR;
                            if (a * PR >= m) break;
                            double acc = 0.;
#pragma unroll
                            for (int bb = 0; bb < GJTile<TR, NT>::CT; ++bb) {
                                const int j = cj + bb * kGJCols;
                                if (j < m) acc = fma(static_cast<double>(R[a][bb]), r64[j], acc);
                            }
#pragma unroll
                            for (int o = 8; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
                            if (cj == 0 && i < m) x[i] += acc;
                        }
                        __syncthreads();
                    }
                }
                mark(kPhaseRefine);
            }
          }
        } else {
            // (S3) LU without pivoting of the free block A[0:m][0:m]; the right-hand
            //      side in column m is eliminated with it.  Right-looking, panels of
            //      kPanel columns, two CTA barriers per panel:
            //      phase 1 - warp 0 applies panel k to the next panel's diagonal rows
            //                (its U12 tile goes to a stage) and factors the next
            //                diagonal block; the other warps apply panel k to the rows
            //                below it and to every other column tile;
            //      phase 2 - the stage is copied into A and all threads solve the next
            //                panel's L21 rows (one row per thread).
            //      Multipliers are stored scaled; rpiv keeps the reciprocal pivots.
            if (m > 0) {
                if (warp == 0) factor_diag(A, ldA, m, 0, rpiv, lane, &s_flag);
                __syncthreads();
                solve_l21(A, ldA, m, 0, rpiv, min(kPanel, m), tid, NT);
                __syncthreads();
                for (int k0 = 0; k0 < m; k0 += kPanel) {
                    const int kb = min(kPanel, m - k0);
                    const int r0 = k0 + kb;
                    const int nct = (m + 1 - r0 + 7) / 8;  // column tiles of [r0, m], rhs included
                    const int top = min(r0 + kPanel, m);   // rows of the next diagonal block
                    if (warp == 0) {
                        update_tile<kU12ToStage>(A, ldA, m, k0, kb, r0, r0, top, stage, lane);
                        mark(kPhaseLUDiag);
                        if (r0 < m) {
                            __syncwarp();
                            factor_diag(A, ldA, m, r0, rpiv, lane, &s_flag);
                        }
                        mark(kPhaseLUPanel);
                    } else {
                        // unit 0: tile 0 below the next diagonal block; unit u >= 1: tile u
                        for (int u = warp - 1; u < nct; u += NW - 1) {
                            if (u == 0) {
                                if (top < m)
                                    update_tile<kU12InRegs>(A, ldA, m, k0, kb, r0, top, m, nullptr, lane);
                            } else {
                                update_tile<kU12InPlace>(A, ldA, m, k0, kb, r0 + 8 * u, r0, m, nullptr, lane);
                            }
                        }
                    }
                    __syncthreads();
                    mark(kPhaseFactor);
                    if (tid < 64) {  // tile 0 of U12 (rows k0+1 .. k0+kb-1) from the stage
                        const int j = tid >> 3, c = r0 + (tid & 7);
                        if (j >= 1 && j < kb && c <= m) A[(k0 + j) * ldA + c] = static_cast<TR>(stage[tid]);
                    }
                    if (top < m) solve_l21(A, ldA, m, r0, rpiv, top, tid, NT);
                    __syncthreads();
                    mark(kPhaseIntEpilogue);
                }
            }
            // (S4) back substitution U x = y (y in column m): every warp inverts some
            //      diagonal blocks, then warp 0 substitutes block by block.
            if (drive) {  // second right-hand side (column m + 1) before U's blocks are inverted
                if (warp == 0 && m > 0) solve_factored_column(A, ldA, m, m + 1, rpiv, lane);
                __syncthreads();
            }
            for (int b = warp; b * kPanel < m; b += NW) invert_diag_block(A, ldA, m, b * kPanel, rpiv, lane);
            __syncthreads();
            if (warp == 0 && m > 0) back_substitute_blocked(A, ldA, m, xs, lane);
            __syncthreads();
            if (drive)
                for (int i = tid; i < m; i += NT) x2[i] = static_cast<double>(A[i * ldA + m + 1]);
            __syncthreads();
        }
        if (drive) {
            // Shaft rotation theta: x = x1 + theta x2 (x1 = (y1, c_r), x2 = (y2, d_r)).
            // The equilibrium rows projected on the test vectors lose every
            // multiplier term (G w = 0 joint by joint), leaving
            //   sum_roots w_r.(b_r - A_r x) + sum_chain w_n.b_n = 0,
            // b_n = -cond (sum of G^T lambda at the node + torque); chain nodes
            // carry no element terms.
            for (int rowi = warp; rowi < 6 * nc; rowi += NW) {
                const int c = rowi / 6, k = rowi % 6;
                const int pr = 6 * pos[KB.con_node[c]];
                double a1 = 0., a2 = 0.;
                for (int j = lane; j < n6; j += 32) {
                    const double arj = static_cast<double>(A[(pr + k) * ldA + j]);
                    a1 += arj * xs[j];
                    a2 += arj * (j < m ? x2[j] : rpiv[j]);
                }
                for (int o = 16; o > 0; o >>= 1) {
                    a1 += __shfl_xor_sync(0xffffffffu, a1, o);
                    a2 += __shfl_xor_sync(0xffffffffu, a2, o);
                }
                if (lane == 0) {
                    con[c * kConStride + conrec::yr + k] = bp[pr + k] - a1;
                    con[c * kConStride + conrec::s2 + k] = a2;
                }
            }
            __syncthreads();
            double* xt = hb + hubsm::xt + 8 * (iter & 1);
            if (tid == 0) {  // this beam's roots: w.s1, w.s2 and G_base^T lambda
                for (int k = 0; k < 8; ++k) xt[k] = 0.;
                for (int c = 0; c < nc; ++c) {
                    const double* cr = con + c * kConStride;
                    for (int k = 0; k < 6; ++k) {
                        xt[0] += cr[conrec::wr + k] * cr[conrec::yr + k];
                        xt[1] += cr[conrec::wr + k] * cr[conrec::s2 + k];
                    }
                    if (is_hub_joint(KB.con_type[c])) joint_base_transpose_add(cr, cr + conrec::lam, xt + 2);
                }
            }
            if (clustered) cluster.sync(); else __syncthreads();
            if (tid == 0) {
                // every CTA sums the beams' parts in rank order, so all find the same theta
                double num = 0., den = 0.;
                double gj[6] = {0., 0., 0., 0., 0., 0.};  // roots' G_base^T lambda
                for (int r = 0; r < KB.model_beams; ++r) {
                    const double* peer = clustered ? cluster.map_shared_rank(xt, r) : xt;
                    num += peer[0];
                    den += peer[1];
                    for (int k = 0; k < 6; ++k) gj[k] += peer[2 + k];
                }
                const double* rv = hb + hubsm::rev;
                double bA[6];
                for (int k = 0; k < 6; ++k) bA[k] = rv[revrec::GtL + k] + (k >= 3 ? rv[revrec::sys + k - 3] : 0.);
                if (hH) {
                    const double* ah = hb + hubsm::ah;
                    joint_base_transpose_add(ah, ah + conrec::lam, bA);
                    for (int k = 0; k < 6; ++k)
                        num -= hb[hubsm::wH + k] * P.conditioner * (ah[conrec::Gl + k] + gj[k]);
                } else {
                    for (int k = 0; k < 6; ++k) bA[k] += gj[k];
                }
                for (int k = 0; k < 6; ++k) num -= hb[hubsm::wA + k] * P.conditioner * bA[k];
                if (!(fabs(den) > 0.)) atomicOr(&s_flag, 2);
                hb[hubsm::theta] = num / den;
            }
            __syncthreads();
            const double th = hb[hubsm::theta];
            for (int i = tid; i < m; i += NT) xs[i] += th * x2[i];
            for (int t = tid; t < 6 * nc; t += NT) {
                const int pr = 6 * pos[KB.con_node[t / 6]];
                xs[pr + t % 6] += th * rpiv[pr + t % 6];
            }
            __syncthreads();
        }
        // (S5) multipliers from the constrained rows: grad^T x_l = b_r - A_r x
        for (int rowi = warp; rowi < 6 * nc; rowi += NW) {
            const int c = rowi / 6, k = rowi % 6;
            const int pr = 6 * pos[KB.con_node[c]];
            double sacc = 0.;
            for (int j = lane; j < n6; j += 32) sacc += static_cast<double>(A[(pr + k) * ldA + j]) * xs[j];
            for (int o = 16; o > 0; o >>= 1) sacc += __shfl_xor_sync(0xffffffffu, sacc, o);
            if (lane == 0) con[c * kConStride + conrec::yr + k] = bp[pr + k] - sacc;
        }
        __syncthreads();
        if (tid < nc) {
            double* cr = con + tid * kConStride;
            const double* y = cr + conrec::yr;
            double yr[3] = {0., 0., 0.};
            if (!solve3(cr + conrec::AX, y + 3, yr)) atomicOr(&s_flag, 2);
            // UnconditionSolution (condition_system.hpp): x_lambda /= conditioner
            for (int k = 0; k < 3; ++k) cr[conrec::xl + k] = y[k] / P.conditioner;
            for (int k = 0; k < 3; ++k) cr[conrec::xl + 3 + k] = yr[k] / P.conditioner;
        }
        __syncthreads();
        if (hub && tid == 0) {
            // this beam's part of the hub rows: sum over its joints of
            // G_base^T (lambda + x_lambda), exchanged over the cluster below
            double* pub = hb + hubsm::pub + 6 * (iter & 1);
            for (int k = 0; k < 6; ++k) pub[k] = 0.;
            for (int c = 0; c < nc; ++c) {
                if (!is_hub_joint(KB.con_type[c])) continue;
                const double* cr = con + c * kConStride;
                double w[6];
                for (int k = 0; k < 6; ++k) w[k] = cr[conrec::lam + k] + cr[conrec::xl + k];
                joint_base_transpose_add(cr, w, pub);
            }
        }
        if (record && KB.dump) {
            const int nl = n6 + 6 * nc;
            double* D = KB.dump + nl * nl + nl;
            for (int t = tid; t < n6; t += NT) D[t] = xs[6 * pos[t / 6] + t % 6];
            if (tid < nc)
                for (int k = 0; k < 6; ++k) D[n6 + 6 * tid + k] = con[tid * kConStride + conrec::xl + k];
        }

        __syncthreads();
        sec_prefetch();  // A is not read again in this iteration
        mark(kPhaseSubstitute);

        // ---- convergence error (calculate_error_sum_squares.hpp:33-79) --------------
        double part = 0.;
        for (int t = tid; t < n6; t += NT) {
            const double pi = xs[6 * pos[t / 6] + t % 6];
            const double xi = sqd[t] * h;
            const double e = pi / (P.atol + P.rtol * fabs(xi));
            part += e * e;
        }
        if (tid < 6 * nc) {
            const double* cr = con + (tid / 6) * kConStride;
            const double pi = cr[conrec::xl + tid % 6];
            const double xi = cr[conrec::lam + tid % 6];
            const double e = pi / (P.atol + P.rtol * fabs(xi));
            part += e * e;
        }
        for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
        double* slot = red + (iter & 1) * (NW + 8);
        if (lane == 0) slot[warp] = part;
        __syncthreads();
        if (tid == 0) {
            double s = 0.;
            for (int w2 = 0; w2 < NW; ++w2) s += slot[w2];
            slot[NW] = s;
            slot[NW + 1] = static_cast<double>(s_flag);
        }
        double total, flags;
        if (clustered) {
            cluster.sync();
            total = 0.;
            flags = 0.;
            for (int r = 0; r < KB.model_beams; ++r) {
                const double* peer = cluster.map_shared_rank(slot, r);
                total += peer[NW];
                flags = fmax(flags, peer[NW + 1]);
            }
        } else {
            __syncthreads();
            total = slot[NW];
            flags = slot[NW + 1];
        }
        double xlh[6] = {0., 0., 0., 0., 0., 0.};
        if (hub) {
            // Hub rows have no element terms: G_hub^T x_lh = -G_hub^T lambda_hub -
            // sum_j G_base,j^T (lambda_j + x_lj), summed over the beams in rank order.
            double sum[6] = {0., 0., 0., 0., 0., 0.};
            for (int r = 0; r < KB.model_beams; ++r) {
                const double* peer = clustered ? cluster.map_shared_rank(hb + hubsm::pub + 6 * (iter & 1), r)
                                               : hb + hubsm::pub + 6 * (iter & 1);
                for (int k = 0; k < 6; ++k) sum[k] += peer[k];
            }
            if (drive) {
                // Drive train, from the roots back to the BC: record 2's rows give
                // the rigid joint's multipliers, record 1's rows (with the torque)
                // the revolute's five (least squares on the three rotation rows,
                // consistent once theta balances them), and G_rev,base^T L_rev
                // is what record 0's BC carries.
                double sumA[6];
                if (hH) {
                    const double* ah = hb + hubsm::ah;
                    double L[6];
                    for (int k = 0; k < 3; ++k) L[k] = -sum[k];
                    const double rr[3] = {-sum[3], -sum[4], -sum[5]};
                    if (!solve3(ah + conrec::AX, rr, L + 3)) flags = 1.;
                    for (int k = 0; k < 6; ++k) sumA[k] = 0.;
                    joint_base_transpose_add(ah, L, sumA);
                    for (int k = 0; k < 6; ++k) {
                        const double xl = L[k] - ah[conrec::lam + k];
                        const double e = xl / (P.atol + P.rtol * fabs(ah[conrec::lam + k]));
                        total += e * e;
                        if (tid == NT - 3) hb[hubsm::ah + conrec::xl + k] = xl;
                    }
                } else {
                    for (int k = 0; k < 6; ++k) sumA[k] = sum[k];
                }
                const double* rv = hb + hubsm::rev;
                double g[6];
                for (int k = 0; k < 6; ++k) g[k] = -sumA[k] - (k >= 3 ? rv[revrec::sys + k - 3] : 0.);
                const double* u = rv + revrec::xcz;
                const double* w = rv + revrec::xcy;
                const double a00 = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
                const double a01 = u[0] * w[0] + u[1] * w[1] + u[2] * w[2];
                const double a11 = w[0] * w[0] + w[1] * w[1] + w[2] * w[2];
                const double r0 = -(u[0] * g[3] + u[1] * g[4] + u[2] * g[5]);
                const double r1 = -(w[0] * g[3] + w[1] * g[4] + w[2] * g[5]);
                const double det = a00 * a11 - a01 * a01;
                if (!(fabs(det) > 0.)) flags = 1.;
                const double L[5] = {g[0], g[1], g[2], (a11 * r0 - a01 * r1) / det, (a00 * r1 - a01 * r0) / det};
                for (int k = 0; k < 5; ++k) {
                    const double xl = L[k] - rv[revrec::lam + k];
                    const double e = xl / (P.atol + P.rtol * fabs(rv[revrec::lam + k]));
                    total += e * e;
                    if (tid == NT - 2) hb[hubsm::rev + revrec::xl + k] = xl;
                }
                for (int k = 0; k < 3; ++k) {
                    sum[k] = -L[k];
                    sum[3 + k] = u[k] * L[3] + w[k] * L[4];
                }
                // the chain nodes' terms of the error sum
                const double th = hb[hubsm::theta];
                for (int r = 1; r < chain; ++r) {
                    const double* rec = r == 1 ? hA : hH;
                    const double* c0 = hb + (r == 1 ? hubsm::cA : hubsm::cH);
                    const double* d0 = hb + (r == 1 ? hubsm::nA : hubsm::dH);
                    for (int k = 0; k < 6; ++k) {
                        const double e = (c0[k] + th * d0[k]) / (P.atol + P.rtol * fabs(rec[hubrec::q_delta + k] * h));
                        total += e * e;
                    }
                }
            }
            const double* br = hb + hubsm::bc;
            for (int k = 0; k < 3; ++k) xlh[k] = -br[conrec::lam + k] - sum[k];
            double yr[3] = {0., 0., 0.};
            if (!solve3(br + conrec::AX, sum + 3, yr)) flags = 1.;
            for (int k = 0; k < 3; ++k) xlh[3 + k] = -br[conrec::lam + 3 + k] - yr[k];
            // the hub's own terms of the error sum (every CTA adds the same values)
            const double* xh = hb + hubsm::xh;
            const double* hqd = hb + hubrec::q_delta;
            for (int k = 0; k < 6; ++k) {
                const double e1 = xh[k] / (P.atol + P.rtol * fabs(hqd[k] * h));
                const double e2 = xlh[k] / (P.atol + P.rtol * fabs(br[conrec::lam + k]));
                total += e1 * e1 + e2 * e2;
            }
        }
        const double err = sqrt(total / static_cast<double>(KB.model_dofs));
        if (KB.rank == 0 && tid == 0 && iter < kMaxNewtonIters) KB.conv[iter] = err;
        iters = iter + 1;

        // ---- update (update_dynamic_prediction.hpp, calculate_displacement.hpp,
        //      update_lambda_prediction.hpp) ----------------------------------------------
        for (int t = tid; t < n6; t += NT) {
            const double delta = xs[6 * pos[t / 6] + t % 6];
            sqd[t] += delta / h;
            if (P.dynamic) {
                sv[t] += P.gamma_prime * delta;
                svd[t] += P.beta_prime * delta;
            }
        }
        if (tid < 6 * nc) {
            double* cr = con + (tid / 6) * kConStride;
            cr[conrec::lam + tid % 6] += cr[conrec::xl + tid % 6];
        }
        if (hub && tid == NT - 1) {
            const double* xh = hb + hubsm::xh;
            for (int k = 0; k < 6; ++k) {
                hb[hubrec::q_delta + k] += xh[k] / h;
                if (P.dynamic) {
                    hb[hubrec::v + k] += P.gamma_prime * xh[k];
                    hb[hubrec::vd + k] += P.beta_prime * xh[k];
                }
                hb[hubsm::bc + conrec::lam + k] += xlh[k];
            }
        }
        if (drive && (tid == NT - 2 || tid == NT - 3) && chain_rec()) {
            double* my_rec = chain_rec();
            const double th = hb[hubsm::theta];
            const double* c0 = hb + (tid == NT - 2 ? hubsm::cA : hubsm::cH);
            const double* d0 = hb + (tid == NT - 2 ? hubsm::nA : hubsm::dH);
            for (int k = 0; k < 6; ++k) {
                const double x = c0[k] + th * d0[k];
                my_rec[hubrec::q_delta + k] += x / h;
                if (P.dynamic) {
                    my_rec[hubrec::v + k] += P.gamma_prime * x;
                    my_rec[hubrec::vd + k] += P.beta_prime * x;
                }
            }
            if (tid == NT - 2)
                for (int k = 0; k < 5; ++k) hb[hubsm::rev + revrec::lam + k] += hb[hubsm::rev + revrec::xl + k];
            else
                for (int k = 0; k < 6; ++k) hb[hubsm::ah + conrec::lam + k] += hb[hubsm::ah + conrec::xl + k];
        }
        __syncthreads();
        displacement();
        __syncthreads();
        mark(kPhaseUpdate);

        if (flags != 0.) {
            status = KYN_ERR_SINGULAR;
            break;
        }
        if (!(err == err) || isinf(err)) {
            status = KYN_ERR_NONFINITE;
            break;
        }
        if (err <= 1.) {
            if (extra < P.refine_iters) {
                ++extra;  // one more correction from the FP64 residual
                continue;
            }
            status = KYN_OK;
            break;
        }
    }

    // the copy issued in the last iteration lands before the region is released
    while (sec_waited < sec_issued) sec_wait();
    __syncthreads();
    if (s_flag & 8) status = KYN_ERR_CUDA;  // a section copy did not complete in time

    // ---- post-step (step.hpp:86-121) ---------------------------------------------------
    if (status == KYN_OK) {
        const double fac = (1. - P.alpha_f) / (1. - P.alpha_m);
        for (int t = tid; t < n6; t += NT) sa[t] += fac * svd[t];
    }
    if (hub && chain_rec()) {
        double* r = chain_rec();
        if (status == KYN_OK) {
            const double fac = (1. - P.alpha_f) / (1. - P.alpha_m);
            for (int k = 0; k < 6; ++k) r[hubrec::a + k] += fac * r[hubrec::vd + k];
            const double* x0 = r + hubrec::x0;
            for (int c = 0; c < 3; ++c) r[hubrec::x + c] = x0[c] + r[hubrec::q + c];
            quat_compose(r + hubrec::q + 3, x0 + 3, r + hubrec::x + 3);
        }
        const double* lam = (tid == NT - 1) ? hb + hubsm::bc + conrec::lam
                           : (tid == NT - 2) ? hb + hubsm::rev + revrec::lam : hb + hubsm::ah + conrec::lam;
        for (int k = 0; k < 6; ++k) r[hubrec::lambda + k] = (tid == NT - 2 && k == 5) ? 0. : lam[k];
    }
    __syncthreads();
    if (hub)  // every beam keeps its copy of the hub state (the input is the caller's)
        for (int k = tid; k < (drive ? chain : 1) * kHubDoubles; k += NT) {
            const int r = k / kHubDoubles, e = k % kHubDoubles;
            const double* src = r == 0 ? hb : r == 1 ? hA : hH;
            if (e < hubrec::input || e >= hubrec::input + 7) slab[L.hub + k] = src[e];
        }
    for (int k = tid; k < N * 7; k += NT) {
        slab[L.q + k] = sq[k];
        slab[L.q_prev + k] = sqp[k];
    }
    for (int k = tid; k < N * 6; k += NT) {
        slab[L.v + k] = sv[k];
        slab[L.vd + k] = svd[k];
        slab[L.a + k] = sa[k];
        slab[L.q_delta + k] = sqd[k];
    }
    if (status == KYN_OK) {
        for (int n = tid; n < N; n += NT) {
            const double* x0 = slab + L.x0 + n * 7;
            for (int c = 0; c < 3; ++c) slab[L.x + n * 7 + c] = x0[c] + sq[n * 7 + c];
            double r[4];
            quat_compose(sq + n * 7 + 3, x0 + 3, r);
            for (int c = 0; c < 4; ++c) slab[L.x + n * 7 + 3 + c] = r[c];
        }
    }
    for (int k = tid; k < N * 9; k += NT) slab[L.tangent + k] = sT[k];
    if (tid < 6 * nc) {
        const double* cr = con + (tid / 6) * kConStride;
        slab[L.lambda + tid] = cr[conrec::lam + tid % 6];
    }
    if (KB.rank == 0 && tid == 0) {
        status_out[KB.plan_model] = status;
        iters_out[KB.plan_model] = iters;
    }
    __syncthreads();
    mark(kPhaseStore);
    if (timing && tid == 0)
        for (int k = 0; k < kNumPhases; ++k) atomicAdd(KB.prof + k, s_ph[k]);
    if (clustered) cluster.sync();  // peers may still read this CTA's slot
}

}  // namespace kyn
