// kyn_capi.cu -- C ABI of the B200 beam path (declared in include/kynema_b200.h).
//
// A context owns a CUDA stream, the resident state of every admitted model and
// cached launch plans.  A step over a list of models launches the fused step
// kernel once per bucket of beams: beams are grouped by cluster size (beams per
// model) and by shared-memory class, and each bucket runs on its own stream so
// the buckets share the GPU.  There is no CPU fallback: without a device every
// entry point fails with KYN_ERR_NO_DEVICE.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <map>
#include <unordered_map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/kynema_b200.h"
#include "kyn_host.hpp"
#include "kyn_step_kernel.cuh"
#include "kyn_types.h"

using namespace kyn;

namespace {

constexpr int kMaxDynSmem = 232448 - 1024;  // 227 KB per CTA on sm_100, minus static use
constexpr int kSmemPerSM = 233472;      // 228 KB per SM
constexpr int kBucketStreams = 8;

struct DevModel {
    HostModel host;
    std::vector<double*> d_slab;     // per beam
    std::vector<int> nt;             // per beam: threads per CTA of the step kernel
    // Per-model values every plan needs, computed once (plans are rebuilt
    // whenever the model set changes, every iteration of a serving loop).
    std::vector<SlabLayout> lay;     // per beam slab layout
    std::vector<KBeam> kt;           // per beam launch record (plan fields filled per plan)
    KBeam* d_kt = nullptr;           // the same records resident on the device (plans gather them)
    std::vector<int> node_base;      // per beam: first global node when its nodes are contiguous, else -1
    int def_nt[2] = {0, 0};          // default threads per CTA, FP64 / FP32 form
    int tuned_nt[2] = {0, 0};        // tuned threads per CTA (0: none), cached per form
    int tuned_sv[2] = {-1, -1};      // tuned free-block solver (-1: the context's), cached per form
    unsigned long long tuned_gen[2] = {~0ull, ~0ull};  // tuned-table generation of that cache
    int lump = 0;                    // kernel kind: 0 beams, 1 with masses / springs /
                                     // drive train (LUMP instance), 2 dense model
    int smem_nt[2][3] = {};          // dynamic smem for 128 / 256 / 512 threads, per form
    double work = 0.;                // largest beam's N^2 Q + 72 (N-1)^3 (ordering in buckets)
    double* d_conv = nullptr;        // [kMaxNewtonIters]
    double* d_dump = nullptr;        // per-beam system dumps (recording mode)
    std::vector<size_t> dump_off;    // per beam offset into d_dump (doubles)
    size_t bytes = 0;
    int last_status = KYN_OK;
    int last_iters = 0;
};

// One model of a plan being built; bucket key: (point masses/springs, cluster
// size, threads, CTAs per SM class); larger work first.
struct Entry {
    int model_index;
    int cluster;
    int nt;
    int cls;
    int smem;
    double work;
    DevModel* m;
    int lump;
    int solver;  // KYN_SOLVER_* of the free-block solve (tuned per size class, or the context's)
};

struct ClassKey {
    int beams, N, Q, nc, precision;
    bool operator<(const ClassKey& o) const {
        if (beams != o.beams) return beams < o.beams;
        if (N != o.N) return N < o.N;
        if (Q != o.Q) return Q < o.Q;
        if (nc != o.nc) return nc < o.nc;
        return precision < o.precision;
    }
};

struct Bucket {
    int cluster = 1;
    int nt = 256;      // threads per CTA (step_kernel instance)
    int lump = 0;      // kernel kind (DevModel::lump)
    int solver = KYN_SOLVER_PANEL_LU;  // free-block solve of this bucket's launch
    int smem = 0;
    int first = 0;     // first beam in the plan's beam array
    int count = 0;     // beams
};

struct Plan {
    std::vector<int> ids;
    int precision = KYN_PRECISION_FP64;
    std::vector<Bucket> buckets;
    KBeam* d_kbeams = nullptr;
    int* d_status = nullptr;      // [nmodels]
    int* d_iters = nullptr;
    int* h_status = nullptr;      // pinned
    int* h_iters = nullptr;
    int nbeams = 0;
    bool record = false;
    unsigned long long epoch = 0;     // model-destroy count when built
    cudaGraphExec_t graph = nullptr;  // captured step (KYN_OPT_CUDA_GRAPH)
    StepCoeffs graph_coeffs{};        // coefficients baked into the captured launches
    ~Plan() {  // buffers belong to the context's plan pool
        if (graph) cudaGraphExecDestroy(graph);
    }
};

// One beam of a batched host<->device transfer.
struct XferBeam {
    double* slab_field;   // slab + field offset
    long long ext_off;    // offset of this beam's first row in the external array
    int map_off;          // offset into the node map; -1: rows in order (ext row k = slab row k)
    int N;
};

// Source of one plan record: a model's resident KBeam and the plan's own fields.
struct PlanSrc {
    const KBeam* src;
    double* dump;
    int plan_model;
    int pad;
};
static_assert(sizeof(KBeam) % 8 == 0, "KBeam is copied in 8-byte words");

// Fills a plan's KBeam array from the models' resident records (one warp per
// record), so that a new plan uploads 24 bytes per beam instead of the record.
__global__ void gather_kbeams(const PlanSrc* __restrict__ srcs, int n, KBeam* __restrict__ out,
                              unsigned long long* prof) {
    const int w = static_cast<int>((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (w >= n) return;
    const PlanSrc sr = srcs[w];
    const unsigned long long* a = reinterpret_cast<const unsigned long long*>(sr.src);
    unsigned long long* b = reinterpret_cast<unsigned long long*>(out + w);
    constexpr int kWords = static_cast<int>(sizeof(KBeam) / 8);
    for (int k = lane; k < kWords; k += 32) b[k] = a[k];
    __syncwarp();
    if (lane == 0) {
        out[w].plan_model = sr.plan_model;
        out[w].dump = sr.dump;
        out[w].prof = prof;
    }
}

struct XferPlan {
    std::vector<int> ids;
    unsigned long long epoch = 0;  // model-destroy count when built
    int kind = -1;        // load channel (0/1) or 100 + state field
    int width = 0;
    long long total = 0;  // doubles in the external array
    XferBeam* d_beams = nullptr;
    int* d_map = nullptr;
    size_t beams_cap = 0, map_cap = 0;  // device buffers are reused when a slot is rebuilt
    int nbeams = 0;
    ~XferPlan() {
        if (d_beams) cudaFree(d_beams);
        if (d_map) cudaFree(d_map);
    }
};

// Copies rows between the external array and the beams' slabs.
// to_slab != 0: external -> slab (loads); else slab -> external (state read).
__global__ void xfer_kernel(const XferBeam* __restrict__ beams, const int* __restrict__ map,
                            double* ext, int width, int to_slab) {
    const XferBeam b = beams[blockIdx.x];
    const int n = b.N * width;
    for (int t = threadIdx.x; t < n; t += blockDim.x) {
        const int k = t / width, c = t - k * width;
        const int row = (b.map_off < 0) ? k : map[b.map_off + k];
        const long long e = b.ext_off + static_cast<long long>(row) * width + c;
        if (to_slab) b.slab_field[t] = ext[e];
        else ext[e] = b.slab_field[t];
    }
}

}  // namespace

struct kyn_ctx {
    int device = 0;
    size_t budget = 0;
    size_t used = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t bstream[kBucketStreams] = {};
    cudaEvent_t fork = nullptr;
    cudaEvent_t join[kBucketStreams] = {};
    std::unordered_map<int, std::unique_ptr<DevModel>> models;
    std::vector<DevModel*> by_id;         // model id -> model (ids are dense and never reused)
    std::vector<Entry> plan_entries_tmp, plan_sorted_tmp;  // plan build buffers (reused)
    std::vector<uint64_t> plan_keys_tmp;
    unsigned long long tuned_gen = 0;     // bumped whenever the tuned table changes
    int next_id = 0;
    std::string err;
    bool record = false;
    std::unique_ptr<Plan> plan;           // last launch plan (cache)
    std::vector<int> pending;             // models of the last kyn_step_async
    int smem_configured = 0;
    bool use_graph = false;               // KYN_OPT_CUDA_GRAPH
    int solver = KYN_SOLVER_PANEL_LU;     // KYN_OPT_LINEAR_SOLVER
    int bulk_sections = 1;                // KYN_OPT_BULK_SECTIONS
    double* h_stage = nullptr;            // pinned staging for loads
    size_t h_stage_len = 0;
    std::unique_ptr<XferPlan> xfer[4];    // cached transfer plans
    std::vector<XferBeam> xfer_beams_tmp; // host build buffers of transfer plans (reused)
    std::vector<int> xfer_map_tmp;
    double* d_stage = nullptr;            // device staging for batched transfers
    size_t d_stage_len = 0;
    int64_t launches = 0;                 // kernels launched so far
    int64_t allocations = 0;              // device and pinned allocations so far
    int64_t last_buckets = 0;
    unsigned long long* d_prof = nullptr; // phase timing counters (KYN_OPT_PHASE_TIMING)
    unsigned long long* d_diag = nullptr; // solve counters (kDiag*, KYN_STAT_SOLVE_*)
    std::map<ClassKey, int> tuned;        // threads per CTA chosen by kyn_autotune
    std::map<ClassKey, int> tuned_solver; // free-block solver chosen by kyn_autotune (FP64 form)
    // Plan buffers, grown on demand and reused by every plan (one step in
    // flight at a time), so rebuilding a plan for a changed model set (the
    // serving loop does it every iteration) allocates nothing in steady state.
    KBeam* pool_kbeams = nullptr;
    size_t pool_kbeams_cap = 0;
    PlanSrc* pool_hsrc = nullptr;         // pinned staging of the plan's record sources
    size_t pool_hsrc_cap = 0;
    PlanSrc* pool_dsrc = nullptr;         // the same on the device
    size_t pool_dsrc_cap = 0;
    unsigned long long destroy_epoch = 0; // models destroyed so far (cached plans check it)
    cudaEvent_t plan_uploaded = nullptr;  // the staging buffer's last upload
    bool plan_upload_pending = false;
    int* pool_status = nullptr;           // device [2][cap]: status, iterations
    int* pool_hstatus = nullptr;          // pinned [2][cap]
    size_t pool_status_cap = 0;
    std::vector<int> presc_ids;           // batched prescribed motion: cached targets
    unsigned long long presc_epoch = 0;   // model-destroy count when they were built
    double** presc_targets = nullptr;     // device [count] slab addresses of con_input slots
    int* presc_vidx = nullptr;            // device [count] row of the caller's array per target
    int presc_rows = 0;                   // constraint rows of the cached id list
    size_t presc_cap = 0;
    int presc_count = 0;
};

namespace {

int set_err(kyn_ctx* c, int code, const std::string& msg) {
    if (c) c->err = msg;
    return code;
}

#define KYN_CUDA(ctx, call)                                                              \
    do {                                                                                 \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess)                                                           \
            return set_err((ctx), KYN_ERR_CUDA,                                          \
                           std::string(#call) + ": " + cudaGetErrorString(e_));          \
    } while (0)

// A device or pinned-host allocation by the context, counted for
// KYN_STAT_ALLOCATIONS.
#define KYN_ALLOC(ctx, call)        \
    do {                            \
        (ctx)->allocations++;       \
        KYN_CUDA(ctx, call);        \
    } while (0)

DevModel* find_model(kyn_ctx* c, int id) {
    return (id >= 0 && static_cast<size_t>(id) < c->by_id.size()) ? c->by_id[id] : nullptr;
}

void register_model(kyn_ctx* c, int id, std::unique_ptr<DevModel> m) {
    if (c->by_id.size() <= static_cast<size_t>(id)) c->by_id.resize(static_cast<size_t>(id) + 1, nullptr);
    c->by_id[id] = m.get();
    c->models[id] = std::move(m);
}

StepCoeffs make_coeffs(const kyn_ctx* c, const kyn_step_params* p) {
    StepCoeffs P{};
    P.solver = c->solver;
    P.diag = c->d_diag;
    P.bulk_sections = c->bulk_sections;
    const bool fp32 = p->precision == KYN_PRECISION_FP32_REFINED;
    P.refine_sweeps = fp32 ? kRefineSweeps : 0;
    P.refine_tol = fp32 ? kRefineTol : 0.;
    const double rho = p->rho_inf;
    P.h = p->h;
    P.alpha_m = (2. * rho - 1.) / (rho + 1.);
    P.alpha_f = rho / (rho + 1.);
    P.gamma = 0.5 + P.alpha_f - P.alpha_m;
    P.beta = 0.25 * (P.gamma + 0.5) * (P.gamma + 0.5);
    P.dynamic = p->is_dynamic_solve ? 1 : 0;
    P.gamma_prime = P.dynamic ? P.gamma / (P.h * P.beta) : 0.;
    P.beta_prime = P.dynamic ? (1. - P.alpha_m) / (P.h * P.h * P.beta * (1. - P.alpha_f)) : 0.;
    P.conditioner = P.beta * P.h * P.h;
    P.atol = p->absolute_convergence_tol;
    P.rtol = p->relative_convergence_tol;
    P.max_iter = std::min<int>(p->max_iter, kMaxNewtonIters);
    P.refine_iters = (p->precision == KYN_PRECISION_FP32_REFINED)
                         ? std::max(0, std::min<int>(p->refine_iters, 4)) : 0;
    return P;
}

// Default threads per CTA for a beam: 256 when two such CTAs fit on an SM
// (their serial phases overlap), else 512 so the one resident CTA has 16
// warps.  kyn_autotune replaces the default per size class by measurement.
int beam_threads(int N, int Q, int nc, int real_bytes, int hub = 0) {
    const int s256 = make_smem(N, Q, nc, real_bytes, 256, hub).bytes;
    return (2 * (s256 + 1024) <= kSmemPerSM) ? 256 : 512;
}

// Registers per thread of an instance: the budget its launch bounds give,
// rounded down to the allocation granule of 8.
int step_regs(int real_bytes, int nt) {
    const int r = 65536 / (nt * step_min_blocks(real_bytes, nt));
    return std::min(255, r & ~7);
}

int beam_smem(int N, int Q, int nc, int real_bytes, int nt, int hub = 0) {
    return make_smem(N, Q, nc, real_bytes, nt, hub).bytes;
}

// Resident CTAs per SM for an instance and shared-memory size.
int ctas_per_sm(int real_bytes, int nt, int smem) {
    const int by_regs = 65536 / (step_regs(real_bytes, nt) * nt);
    const int per = smem + 1024;
    return std::max(1, std::min(by_regs, kSmemPerSM / per));
}

// Hub record kind of a model for make_smem: 0 none, 1 a hub, 2 a drive train.
int hub_kind(const HostModel& h) {
    return h.chain.size() > 1 ? 2 : h.hub >= 0 ? 1 : 0;
}

// Size class of a model for the tuned thread-count table.
ClassKey class_key(const HostModel& h, int precision) {
    ClassKey k{static_cast<int>(h.beams.size()), 0, 0, 0, precision};
    for (const HostBeam& b : h.beams) {
        k.N = std::max(k.N, b.N);
        k.Q = std::max(k.Q, b.Q);
        k.nc = std::max(k.nc, b.nc);
    }
    return k;
}

// Dynamic shared memory of a dense model's CTA.
int dense_smem(const HostModel& H, const HostBeam& hb, int nt) {
    return make_dense_smem(hb.N, H.ndofs, nt, hb.comp_maxN, hb.comp_maxQ, hb.cond_nd, hb.cond_md_off >= 0).bytes;
}

// Fills the per-model values that plans and transfer plans reuse.
void prepare_model(DevModel* m) {
    const HostModel& H = m->host;
    const int hubf = hub_kind(H);
    m->lay.clear();
    m->kt.clear();
    m->work = 0.;
    // masses, springs, drive trains and dense models run in the LUMP instance
    bool lump = H.chain.size() > 1;
    for (const HostBeam& hb : H.beams) lump |= hb.n_mass + hb.n_spring > 0;
    m->lump = (!H.beams.empty() && H.beams[0].dense) ? 2 : lump ? 1 : 0;
    for (int f = 0; f < 2; ++f) {
        const int rb = f ? 4 : 8;
        m->def_nt[f] = 128;
        for (int k = 0; k < 3; ++k) m->smem_nt[f][k] = 0;
        for (const HostBeam& hb : H.beams) {
            if (hb.dense) {  // the dense bordered system, FP64 in both forms
                for (int k = 0; k < 3; ++k)
                    m->smem_nt[f][k] = std::max(
                        m->smem_nt[f][k],
                        dense_smem(H, hb, 128 << k));
                // 128 threads, or for a condensed model (elements assembled and
                // eliminated one after the other in one CTA) the most that fit
                if (hb.cond_nd > 0)
                    for (int nt : {512, 256})
                        if (dense_smem(H, hb, nt) <= kMaxDynSmem) {
                            m->def_nt[f] = nt;
                            break;
                        }
                continue;
            }
            m->def_nt[f] = std::max(m->def_nt[f], beam_threads(hb.N, hb.Q, hb.nc, rb, hubf));
            for (int k = 0; k < 3; ++k)
                m->smem_nt[f][k] = std::max(m->smem_nt[f][k], beam_smem(hb.N, hb.Q, hb.nc, rb, 128 << k, hubf));
        }
    }
    m->node_base.clear();
    for (const HostBeam& hb : H.beams) {
        int base = hb.node_ids.empty() ? -1 : hb.node_ids[0];
        for (int k = 0; k < hb.N && base >= 0; ++k)
            if (hb.node_ids[k] != base + k) base = -1;
        m->node_base.push_back(base);
    }
    for (size_t b = 0; b < H.beams.size(); ++b) {
        const HostBeam& hb = H.beams[b];
        m->lay.push_back(make_slab_layout(hb.N, hb.Q));
        const double N = hb.N, Q = hb.Q;
        m->work = std::max(m->work, N * N * Q + 72. * (N - 1) * (N - 1) * (N - 1));
        KBeam k{};
        k.slab = m->d_slab[b];
        k.N = hb.N;
        k.Q = hb.Q;
        k.nc = hb.nc;
        k.rank = static_cast<int>(b);
        k.model_beams = static_cast<int>(H.beams.size());
        k.model_dofs = H.ndofs;
        for (int s2 = 0; s2 < kMaxBeamConstraints; ++s2) {
            k.con_node[s2] = hb.con_node[s2];
            k.con_type[s2] = hb.con_type[s2];
            k.con_row[s2] = hb.con_row[s2];
            for (int d = 0; d < 3; ++d) k.con_X0[s2][d] = hb.con_X0[s2][d];
            for (int d = 0; d < 3; ++d) k.con_axis[s2][d] = hb.con_axis[s2][d];
        }
        for (int d = 0; d < 3; ++d) k.gravity[d] = H.gravity[d];
        k.lumped = (hb.n_mass + hb.n_spring > 0) ? m->d_slab[b] + hb.lumped_off : nullptr;
        k.n_mass = hb.n_mass;
        k.n_spring = hb.n_spring;
        k.conv = m->d_conv;
        k.hub = static_cast<int>(H.chain.size());
        k.hub_con_type = H.hub_con_type;
        k.dense = hb.dense ? 1 : 0;
        k.n_comps = hb.n_comps;
        k.comps = hb.n_comps > 0 ? m->d_slab[b] + hb.comps_off : nullptr;
        k.comp_maxN = hb.comp_maxN;
        k.comp_maxQ = hb.comp_maxQ;
        k.cond_nd = hb.cond_nd;
        k.cond_md = hb.cond_md_off >= 0 ? m->d_slab[b] + hb.cond_md_off : nullptr;
        k.con_frames = hb.frames_off >= 0 ? m->d_slab[b] + hb.frames_off : nullptr;
        for (int s2 = 0; s2 < kMaxBeamConstraints; ++s2) k.con_base[s2] = hb.con_base[s2];
        m->kt.push_back(k);
    }
}

int nt_index(int nt) { return nt == 128 ? 0 : nt == 256 ? 1 : 2; }

// The model's launch records, resident on the device for the plans to gather
// (stream-ordered; the host copy m->kt stays alive with the model).
int upload_templates(kyn_ctx* c, DevModel* m) {
    const size_t len = sizeof(KBeam) * m->kt.size();
    KYN_ALLOC(c, cudaMallocAsync(reinterpret_cast<void**>(&m->d_kt), len, c->stream));
    KYN_CUDA(c, cudaMemcpyAsync(m->d_kt, m->kt.data(), len, cudaMemcpyHostToDevice, c->stream));
    m->bytes += len;
    c->used += len;
    return KYN_OK;
}

// Per-call device buffers grow by doubling from a floor sized for a serving
// batch, stream-ordered on the context stream (no device synchronisation: work
// already queued on the stream still reads the old buffer before it is freed).
template <typename T>
int grow_device(kyn_ctx* c, T*& p, size_t& cap, size_t need, size_t floor) {
    if (cap >= need && p) return KYN_OK;
    size_t nc = std::max(cap, floor);
    while (nc < need) nc *= 2;
    if (p) KYN_CUDA(c, cudaFreeAsync(p, c->stream));
    p = nullptr;
    KYN_ALLOC(c, cudaMallocAsync(reinterpret_cast<void**>(&p), sizeof(T) * nc, c->stream));
    cap = nc;
    return KYN_OK;
}

// Pinned host staging grows the same way; cudaMallocHost is slow, so growth
// events are kept rare.  Copies from the old buffer are finished first.
template <typename T>
int grow_pinned(kyn_ctx* c, T*& p, size_t& cap, size_t need, size_t floor) {
    if (cap >= need && p) return KYN_OK;
    size_t nc = std::max(cap, floor);
    while (nc < need) nc *= 2;
    if (p) {
        KYN_CUDA(c, cudaStreamSynchronize(c->stream));
        KYN_CUDA(c, cudaFreeHost(p));
    }
    p = nullptr;
    KYN_ALLOC(c, cudaMallocHost(reinterpret_cast<void**>(&p), sizeof(T) * nc));
    cap = nc;
    return KYN_OK;
}

constexpr size_t kPoolBeams = 16384;     // growth floor of the per-beam buffers
constexpr size_t kPoolRows = 16384 * 24; // growth floor of the per-node-row buffers

// Builds (or reuses) the launch plan for this id list.
int get_plan(kyn_ctx* c, const int* ids, int n, int precision, Plan** out) {
    if (c->plan && c->plan->record == c->record && c->plan->precision == precision &&
        c->plan->epoch == c->destroy_epoch && static_cast<int>(c->plan->ids.size()) == n &&
        std::equal(ids, ids + n, c->plan->ids.begin())) {
        *out = c->plan.get();
        return KYN_OK;
    }
    auto plan = std::make_unique<Plan>();
    plan->epoch = c->destroy_epoch;
    plan->ids.assign(ids, ids + n);
    plan->record = c->record;
    plan->precision = precision;
    const int f = (precision == KYN_PRECISION_FP32_REFINED) ? 1 : 0;
    const int rbytes = f ? 4 : 8;
    std::vector<Entry>& all = c->plan_entries_tmp;
    all.clear();
    all.reserve(n);
    std::vector<uint64_t>& keys = c->plan_keys_tmp;
    keys.clear();
    keys.reserve(n);
    if (n >= (1 << 26)) return set_err(c, KYN_ERR_UNSUPPORTED, "more than 2^26 models in one step");
    size_t nbeams = 0;
    for (int i = 0; i < n; ++i) {
        DevModel* m = find_model(c, ids[i]);
        if (!m) return set_err(c, KYN_ERR_NOT_FOUND, "unknown model id in step list");
        int nt = m->def_nt[f];
        if (!c->tuned.empty()) {
            if (m->tuned_gen[f] != c->tuned_gen) {  // per-model cache of the tuned table
                const ClassKey ck = class_key(m->host, precision);
                const auto tuned = c->tuned.find(ck);
                m->tuned_nt[f] = (tuned != c->tuned.end()) ? tuned->second : 0;
                const auto tsv = c->tuned_solver.find(ck);
                m->tuned_sv[f] = (tsv != c->tuned_solver.end()) ? tsv->second : -1;
                m->tuned_gen[f] = c->tuned_gen;
            }
            if (m->tuned_nt[f] > 0) nt = m->tuned_nt[f];
        }
        const int solver = (!c->tuned.empty() && m->tuned_sv[f] >= 0) ? m->tuned_sv[f] : c->solver;
        const int smem = m->smem_nt[f][nt_index(nt)];
        const int cluster = static_cast<int>(m->kt.size());
        const int cls = ctas_per_sm(rbytes, nt, smem);
        all.push_back({i, cluster, nt, cls, smem, m->work, m, m->lump, solver});
        // one 64-bit sort key: kernel kind (beams, masses/springs, dense models),
        // larger clusters first, more threads first, fewer CTAs per SM first,
        // more work first, then model order
        const uint64_t work = static_cast<uint64_t>(std::min(m->work, 1048575.));
        keys.push_back((static_cast<uint64_t>(m->lump) << 62) |
                       (static_cast<uint64_t>(15 - std::min(cluster, 15)) << 58) |
                       (static_cast<uint64_t>(2 - nt_index(nt)) << 56) |
                       (static_cast<uint64_t>(std::min(cls, 15)) << 52) |
                       (static_cast<uint64_t>(solver == KYN_SOLVER_GAUSS_JORDAN ? 1 : 0) << 51) |
                       ((1048575ull - work) << 31) | static_cast<uint64_t>(i));
        nbeams += m->kt.size();
    }
    std::sort(keys.begin(), keys.end());
    std::vector<Entry>& entries = c->plan_sorted_tmp;
    entries.clear();
    entries.reserve(n);
    for (uint64_t k : keys) entries.push_back(all[static_cast<size_t>(k & ((1ull << 31) - 1))]);
    // The record sources go through a pinned staging buffer (one DMA) and a
    // gather on the device; wait for the previous plan's upload before refilling it
    if (c->plan_upload_pending) {
        KYN_CUDA(c, cudaEventSynchronize(c->plan_uploaded));
        c->plan_upload_pending = false;
    }
    {
        const int rc = grow_pinned(c, c->pool_hsrc, c->pool_hsrc_cap, nbeams, kPoolBeams);
        if (rc != KYN_OK) return rc;
    }
    PlanSrc* kb = c->pool_hsrc;
    size_t nk = 0;
    for (size_t e = 0; e < entries.size(); ++e) {
        const Entry& en = entries[e];
        if (plan->buckets.empty() || plan->buckets.back().cluster != en.cluster ||
            plan->buckets.back().nt != en.nt || plan->buckets.back().lump != en.lump ||
            plan->buckets.back().solver != en.solver ||
            ctas_per_sm(rbytes, en.nt, plan->buckets.back().smem) != en.cls) {
            Bucket bk;
            bk.cluster = en.cluster;
            bk.nt = en.nt;
            bk.lump = en.lump;
            bk.solver = en.solver;
            bk.first = static_cast<int>(nk);
            plan->buckets.push_back(bk);
        }
        Bucket& bk = plan->buckets.back();
        bk.smem = std::max(bk.smem, en.smem);
        DevModel* m = en.m;
        for (size_t b = 0; b < m->kt.size(); ++b) {
            PlanSrc& k = kb[nk++];
            k.src = m->d_kt + b;
            k.plan_model = en.model_index;
            // the system dump covers single-node constraints only
            k.dump = (c->record && m->d_dump && !m->kt[b].hub) ? m->d_dump + m->dump_off[b] : nullptr;
            bk.count++;
        }
    }
    plan->nbeams = static_cast<int>(nk);
    {
        int rc = grow_device(c, c->pool_kbeams, c->pool_kbeams_cap, nk, kPoolBeams);
        if (rc != KYN_OK) return rc;
        rc = grow_device(c, c->pool_dsrc, c->pool_dsrc_cap, nk, kPoolBeams);
        if (rc != KYN_OK) return rc;
        if (c->pool_status_cap < static_cast<size_t>(n) || !c->pool_status) {
            // status and iteration counts share one buffer: [cap] + [cap]
            size_t cap = std::max(c->pool_status_cap, kPoolBeams);
            while (cap < static_cast<size_t>(n)) cap *= 2;
            size_t dcap = 0, hcap = 0;
            if (c->pool_status) KYN_CUDA(c, cudaFreeAsync(c->pool_status, c->stream));
            c->pool_status = nullptr;
            rc = grow_device(c, c->pool_status, dcap, 2 * cap, 2 * cap);
            if (rc != KYN_OK) return rc;
            rc = grow_pinned(c, c->pool_hstatus, hcap, 2 * cap, 2 * cap);
            if (rc != KYN_OK) return rc;
            c->pool_status_cap = cap;
        }
    }
    plan->d_kbeams = c->pool_kbeams;
    plan->d_status = c->pool_status;
    plan->d_iters = c->pool_status + c->pool_status_cap;
    plan->h_status = c->pool_hstatus;
    plan->h_iters = c->pool_hstatus + c->pool_status_cap;
    KYN_CUDA(c, cudaMemcpyAsync(c->pool_dsrc, kb, sizeof(PlanSrc) * nk, cudaMemcpyHostToDevice,
                                c->stream));
    KYN_CUDA(c, cudaEventRecord(c->plan_uploaded, c->stream));
    if (nk > 0) {
        const int threads = 256;
        const int blocks = static_cast<int>((nk * 32 + threads - 1) / threads);
        gather_kbeams<<<blocks, threads, 0, c->stream>>>(c->pool_dsrc, static_cast<int>(nk), plan->d_kbeams,
                                                          c->d_prof);
        KYN_CUDA(c, cudaGetLastError());
        c->launches++;
    }
    c->plan_upload_pending = true;
    c->plan = std::move(plan);
    *out = c->plan.get();
    return KYN_OK;
}

using StepKernelFn = void (*)(const KBeam*, StepCoeffs, int, int*, int*);

// The step kernel instance for an arithmetic form, a thread count and the
// kernel kind (0 beams, 1 with point masses / springs / a drive train, 2 a
// dense model, which runs in FP64 in both forms).
StepKernelFn pick_kernel(bool fp32, int nt, int lump, bool gauss_jordan = false) {
    if (lump == 2) return nt == 128 ? dense_kernel<128> : nt == 256 ? dense_kernel<256> : dense_kernel<512>;
    if (!lump && gauss_jordan) {
        if (fp32) return nt == 128 ? step_kernel<float, 128, false, true>
                       : nt == 256 ? step_kernel<float, 256, false, true> : step_kernel<float, 512, false, true>;
        return nt == 128 ? step_kernel<double, 128, false, true>
             : nt == 256 ? step_kernel<double, 256, false, true> : step_kernel<double, 512, false, true>;
    }
    if (lump) {
        if (fp32) return nt == 128 ? step_kernel<float, 128, true>
                       : nt == 256 ? step_kernel<float, 256, true> : step_kernel<float, 512, true>;
        return nt == 128 ? step_kernel<double, 128, true>
             : nt == 256 ? step_kernel<double, 256, true> : step_kernel<double, 512, true>;
    }
    if (fp32) return nt == 128 ? step_kernel<float, 128, false>
                   : nt == 256 ? step_kernel<float, 256, false> : step_kernel<float, 512, false>;
    return nt == 128 ? step_kernel<double, 128, false>
         : nt == 256 ? step_kernel<double, 256, false> : step_kernel<double, 512, false>;
}

template <typename K>
cudaError_t set_smem_attr(K kernel) {
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
}

int configure_smem(kyn_ctx* c) {
    if (c->smem_configured < kMaxDynSmem) {
        for (int k = 0; k < 24; ++k)
            KYN_CUDA(c, set_smem_attr(pick_kernel(k & 1, 128 << ((k >> 1) % 3), (k / 6) % 3, k >= 18)));
        c->smem_configured = kMaxDynSmem;
    }
    return KYN_OK;
}

int launch_plan(kyn_ctx* c, Plan* plan, const kyn_step_params* p) {
    const StepCoeffs P = make_coeffs(c, p);
    int rc = configure_smem(c);
    if (rc != KYN_OK) return rc;
    KYN_CUDA(c, cudaEventRecord(c->fork, c->stream));
    const int nb = static_cast<int>(plan->buckets.size());
    for (int b = 0; b < nb; ++b) {
        const Bucket& bk = plan->buckets[b];
        cudaStream_t s = c->bstream[b % kBucketStreams];
        KYN_CUDA(c, cudaStreamWaitEvent(s, c->fork, 0));
        cudaLaunchConfig_t cfg{};
        cfg.gridDim = dim3(bk.count, 1, 1);
        cfg.blockDim = dim3(bk.nt, 1, 1);
        cfg.dynamicSmemBytes = bk.smem;
        cfg.stream = s;
        cudaLaunchAttribute attr[1];
        if (bk.cluster > 1) {
            attr[0].id = cudaLaunchAttributeClusterDimension;
            attr[0].val.clusterDim.x = bk.cluster;
            attr[0].val.clusterDim.y = 1;
            attr[0].val.clusterDim.z = 1;
            cfg.attrs = attr;
            cfg.numAttrs = 1;
        }
        const KBeam* beams = plan->d_kbeams + bk.first;
        const int rec = plan->record ? 1 : 0;
        const bool fp32 = plan->precision == KYN_PRECISION_FP32_REFINED;
        StepCoeffs Pb = P;
        Pb.solver = bk.solver;
        KYN_CUDA(c, cudaLaunchKernelEx(&cfg, pick_kernel(fp32, bk.nt, bk.lump, bk.solver == KYN_SOLVER_GAUSS_JORDAN),
                                       beams, Pb, rec,
                                       plan->d_status, plan->d_iters));
        c->launches++;
    }
    c->last_buckets = nb;
    for (int b = 0; b < std::min(nb, kBucketStreams); ++b) {
        KYN_CUDA(c, cudaEventRecord(c->join[b], c->bstream[b]));
        KYN_CUDA(c, cudaStreamWaitEvent(c->stream, c->join[b], 0));
    }
    const int n = static_cast<int>(plan->ids.size());
    KYN_CUDA(c, cudaMemcpyAsync(plan->h_status, plan->d_status, sizeof(int) * n,
                                cudaMemcpyDeviceToHost, c->stream));
    KYN_CUDA(c, cudaMemcpyAsync(plan->h_iters, plan->d_iters, sizeof(int) * n,
                                cudaMemcpyDeviceToHost, c->stream));
    return KYN_OK;
}

int finish_plan(kyn_ctx* c, Plan* plan, int* status_out, int* iters_out) {
    KYN_CUDA(c, cudaStreamSynchronize(c->stream));
    const int n = static_cast<int>(plan->ids.size());
    for (int i = 0; i < n; ++i) {
        DevModel* m = find_model(c, plan->ids[i]);
        if (m) {
            m->last_status = plan->h_status[i];
            m->last_iters = plan->h_iters[i];
        }
        if (status_out) status_out[i] = plan->h_status[i];
        if (iters_out) iters_out[i] = plan->h_iters[i];
    }
    return KYN_OK;
}

int field_slot(int field, const SlabLayout& L, int* width) {
    switch (field) {
        case KYN_FIELD_X0: *width = 7; return L.x0;
        case KYN_FIELD_X: *width = 7; return L.x;
        case KYN_FIELD_Q: *width = 7; return L.q;
        case KYN_FIELD_Q_PREV: *width = 7; return L.q_prev;
        case KYN_FIELD_Q_DELTA: *width = 6; return L.q_delta;
        case KYN_FIELD_V: *width = 6; return L.v;
        case KYN_FIELD_VD: *width = 6; return L.vd;
        case KYN_FIELD_A: *width = 6; return L.a;
        case KYN_FIELD_F: *width = 6; return L.f;
        default: return -1;
    }
}

// Offset of a node field inside a slab's hub region (-1: not kept for the hub;
// the hub carries no external load, so its f reads as zero).
int hub_field_offset(int field, int* w) {
    switch (field) {
        case KYN_FIELD_X0: *w = 7; return hubrec::x0;
        case KYN_FIELD_X: *w = 7; return hubrec::x;
        case KYN_FIELD_Q: *w = 7; return hubrec::q;
        case KYN_FIELD_Q_PREV: *w = 7; return hubrec::q_prev;
        case KYN_FIELD_Q_DELTA: *w = 6; return hubrec::q_delta;
        case KYN_FIELD_V: *w = 6; return hubrec::v;
        case KYN_FIELD_VD: *w = 6; return hubrec::vd;
        case KYN_FIELD_A: *w = 6; return hubrec::a;
        default: return -1;
    }
}

// kind: KYN_LOAD_NODE_FX (0), KYN_LOAD_STATE_F (1), or 100 + node field.
int get_xfer(kyn_ctx* c, const int* ids, int n, int kind, XferPlan** out) {
    const int slot = (kind == KYN_LOAD_NODE_FX) ? 0 : (kind == KYN_LOAD_STATE_F) ? 1
                                                     : (kind == 100 + KYN_FIELD_Q) ? 2 : 3;
    auto& cached = c->xfer[slot];
    if (cached && cached->kind == kind && cached->epoch == c->destroy_epoch &&
        static_cast<int>(cached->ids.size()) == n &&
        std::equal(ids, ids + n, cached->ids.begin())) {
        *out = cached.get();
        return KYN_OK;
    }
    // Reuse the slot's device buffers (the id set changes every serving iteration).
    std::unique_ptr<XferPlan> xp = cached ? std::move(cached) : std::make_unique<XferPlan>();
    xp->ids.assign(ids, ids + n);
    xp->epoch = c->destroy_epoch;
    xp->width = 0;
    xp->kind = kind;
    std::vector<XferBeam>& beams = c->xfer_beams_tmp;
    std::vector<int>& map = c->xfer_map_tmp;
    beams.clear();
    map.clear();
    long long off = 0;
    for (int i = 0; i < n; ++i) {
        DevModel* m = find_model(c, ids[i]);
        if (!m) return set_err(c, KYN_ERR_NOT_FOUND, "unknown model id in batch");
        long long elem = 0;
        for (size_t bi = 0; bi < m->host.beams.size(); ++bi) {
            const HostBeam& b = m->host.beams[bi];
            const SlabLayout& L = m->lay[bi];
            XferBeam xb{};
            xb.N = b.N;
            xb.map_off = static_cast<int>(map.size());
            int width = 6, fo;
            if (kind == KYN_LOAD_NODE_FX) {
                if (b.elem_ids.size() != 1 || b.dense)
                    return set_err(c, KYN_ERR_UNSUPPORTED,
                                   "batched node_FX needs single-element beams (use kyn_model_set_loads)");
                fo = L.fx;
                xb.ext_off = off + elem * 6;
                xb.map_off = -1;   // element rows in order
            } else {
                fo = (kind == KYN_LOAD_STATE_F) ? L.f : field_slot(kind - 100, L, &width);
                if (fo < 0) return set_err(c, KYN_ERR_INVALID, "field not available in batch form");
                if (m->node_base[bi] >= 0) {  // the beam's nodes are consecutive model nodes
                    xb.ext_off = off + static_cast<long long>(m->node_base[bi]) * width;
                    xb.map_off = -1;
                } else {
                    xb.ext_off = off;
                    for (int k = 0; k < b.N; ++k) map.push_back(b.node_ids[k]);
                }
            }
            xp->width = width;
            xb.slab_field = m->d_slab[bi] + fo;
            beams.push_back(xb);
            elem += b.N;
        }
        for (size_t r = 0; r < m->host.chain.size() && kind >= 100; ++r) {  // hub rows, from beam 0's copy
            int hw = 0;
            const int ho = hub_field_offset(kind - 100, &hw);
            if (ho < 0) return set_err(c, KYN_ERR_UNSUPPORTED, "field not kept for a hub node");
            const HostBeam& b0 = m->host.beams[0];
            const SlabLayout L0 = make_slab_layout(b0.N, b0.Q);
            XferBeam xb{};
            xb.N = 1;
            xb.map_off = static_cast<int>(map.size());
            xb.ext_off = off;
            xb.slab_field = m->d_slab[0] + L0.hub + static_cast<int>(r) * kHubDoubles + ho;
            map.push_back(m->host.chain[r]);
            beams.push_back(xb);
        }
        off += (kind == KYN_LOAD_NODE_FX) ? elem * 6 : static_cast<long long>(m->host.num_nodes) * xp->width;
    }
    if (xp->width == 0) xp->width = 6;
    xp->total = off;
    xp->nbeams = static_cast<int>(beams.size());
    {
        int rc = grow_device(c, xp->d_beams, xp->beams_cap, beams.size(), kPoolBeams);
        if (rc != KYN_OK) return rc;
        rc = grow_device(c, xp->d_map, xp->map_cap, map.size(), kPoolRows);
        if (rc != KYN_OK) return rc;
    }
    // pageable sources: staged before the calls return; stream order does the rest
    KYN_CUDA(c, cudaMemcpyAsync(xp->d_beams, beams.data(), sizeof(XferBeam) * beams.size(),
                                cudaMemcpyHostToDevice, c->stream));
    KYN_CUDA(c, cudaMemcpyAsync(xp->d_map, map.data(), sizeof(int) * map.size(),
                                cudaMemcpyHostToDevice, c->stream));
    cached = std::move(xp);
    *out = cached.get();
    return KYN_OK;
}

int ensure_stage(kyn_ctx* c, long long doubles) {
    return grow_device(c, c->d_stage, c->d_stage_len, static_cast<size_t>(std::max<long long>(1, doubles)),
                       kPoolRows * 6);
}

}  // namespace

extern "C" {

kyn_ctx* kyn_ctx_create(int device, size_t hbm_budget_bytes) {
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count <= device || device < 0) return nullptr;
    if (cudaSetDevice(device) != cudaSuccess) return nullptr;
    auto* c = new kyn_ctx();
    c->device = device;
    c->budget = hbm_budget_bytes;
    bool ok = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) == cudaSuccess;
    for (int i = 0; i < kBucketStreams && ok; ++i) {
        ok = cudaStreamCreateWithFlags(&c->bstream[i], cudaStreamNonBlocking) == cudaSuccess &&
             cudaEventCreateWithFlags(&c->join[i], cudaEventDisableTiming) == cudaSuccess;
    }
    ok = ok && cudaEventCreateWithFlags(&c->fork, cudaEventDisableTiming) == cudaSuccess;
    ok = ok && cudaEventCreateWithFlags(&c->plan_uploaded, cudaEventDisableTiming) == cudaSuccess;
    if (ok) {
        c->allocations++;
        ok = cudaMalloc(&c->d_diag, kNumDiag * sizeof(unsigned long long)) == cudaSuccess &&
             cudaMemset(c->d_diag, 0, kNumDiag * sizeof(unsigned long long)) == cudaSuccess;
    }
    // Slabs come from the device's stream-ordered pool; keep freed blocks in
    // the pool instead of returning them at each synchronisation, so that
    // models created and destroyed every serving iteration reuse memory.
    cudaMemPool_t pool = nullptr;
    if (ok && cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
        uint64_t keep = ~0ull;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    if (!ok) {
        kyn_ctx_destroy(c);
        return nullptr;
    }
    return c;
}

void kyn_ctx_destroy(kyn_ctx* c) {
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    c->plan.reset();
    for (auto& kv : c->models) {
        for (double* p : kv.second->d_slab) cudaFree(p);
        if (kv.second->d_conv) cudaFree(kv.second->d_conv);
        if (kv.second->d_dump) cudaFree(kv.second->d_dump);
        if (kv.second->d_kt) cudaFree(kv.second->d_kt);
    }
    c->models.clear();
    c->by_id.clear();
    if (c->pool_kbeams) cudaFree(c->pool_kbeams);
    if (c->pool_hsrc) cudaFreeHost(c->pool_hsrc);
    if (c->pool_dsrc) cudaFree(c->pool_dsrc);
    if (c->plan_uploaded) cudaEventDestroy(c->plan_uploaded);
    if (c->pool_status) cudaFree(c->pool_status);
    if (c->pool_hstatus) cudaFreeHost(c->pool_hstatus);
    if (c->presc_targets) cudaFree(c->presc_targets);
    if (c->presc_vidx) cudaFree(c->presc_vidx);
    if (c->h_stage) cudaFreeHost(c->h_stage);
    for (auto& x : c->xfer) x.reset();
    if (c->d_stage) cudaFree(c->d_stage);
    if (c->d_diag) cudaFree(c->d_diag);
    for (int i = 0; i < kBucketStreams; ++i) {
        if (c->bstream[i]) cudaStreamDestroy(c->bstream[i]);
        if (c->join[i]) cudaEventDestroy(c->join[i]);
    }
    if (c->fork) cudaEventDestroy(c->fork);
    if (c->d_prof) cudaFree(c->d_prof);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

const char* kyn_last_error(const kyn_ctx* c) { return c ? c->err.c_str() : "null context"; }

size_t kyn_ctx_used_bytes(const kyn_ctx* c) { return c ? c->used : 0; }

void* kyn_ctx_stream(kyn_ctx* c) { return c ? static_cast<void*>(c->stream) : nullptr; }

int kyn_ctx_stat(kyn_ctx* c, int stat, int64_t* value) {
    if (!c || !value) return KYN_ERR_INVALID;
    if (stat == KYN_STAT_KERNEL_LAUNCHES) *value = c->launches;
    else if (stat == KYN_STAT_STEP_BUCKETS) *value = c->last_buckets;
    else if (stat == KYN_STAT_ALLOCATIONS) *value = c->allocations;
    else if (stat >= KYN_STAT_SOLVES_CHECKED && stat <= KYN_STAT_REFINE_SHORT) {
        static_assert(KYN_STAT_GUARD_TRIPS - KYN_STAT_SOLVES_CHECKED == kDiagGuardTrips &&
                          KYN_STAT_MAX_BACKWARD_ERROR - KYN_STAT_SOLVES_CHECKED == kDiagMaxBackwardError &&
                          KYN_STAT_REFINE_SWEEPS - KYN_STAT_SOLVES_CHECKED == kDiagRefineSweeps &&
                          KYN_STAT_REFINE_SHORT - KYN_STAT_SOLVES_CHECKED == kDiagRefineShort,
                      "KYN_STAT_SOLVE* follow kDiag*");
        unsigned long long v = 0;
        KYN_CUDA(c, cudaStreamSynchronize(c->stream));
        KYN_CUDA(c, cudaMemcpy(&v, c->d_diag + (stat - KYN_STAT_SOLVES_CHECKED), sizeof(v),
                               cudaMemcpyDeviceToHost));
        *value = static_cast<int64_t>(v);
    }
    else if (stat >= KYN_STAT_PHASE_CYCLES && stat < KYN_STAT_PHASE_CYCLES + kNumPhases) {
        if (!c->d_prof) return set_err(c, KYN_ERR_INVALID, "KYN_OPT_PHASE_TIMING is not set");
        unsigned long long v = 0;
        KYN_CUDA(c, cudaStreamSynchronize(c->stream));
        KYN_CUDA(c, cudaMemcpy(&v, c->d_prof + (stat - KYN_STAT_PHASE_CYCLES), sizeof(v),
                               cudaMemcpyDeviceToHost));
        *value = static_cast<int64_t>(v);
    } else return set_err(c, KYN_ERR_INVALID, "unknown statistic");
    return KYN_OK;
}

int kyn_ctx_set_option(kyn_ctx* c, int option, int64_t value) {
    if (!c) return KYN_ERR_INVALID;
    if (option == KYN_OPT_RECORD_SYSTEM) {
        c->record = value != 0;
        if (c->record) {
            for (auto& kv : c->models) {
                DevModel* m = kv.second.get();
                if (m->d_dump) continue;
                size_t tot = 0;
                m->dump_off.clear();
                for (auto& b : m->host.beams) {
                    const size_t nl = 6 * b.N + 6 * b.nc;
                    m->dump_off.push_back(tot);
                    tot += nl * nl + 2 * nl;
                }
                KYN_ALLOC(c, cudaMalloc(&m->d_dump, tot * sizeof(double)));
                KYN_CUDA(c, cudaMemset(m->d_dump, 0, tot * sizeof(double)));
            }
        }
        c->plan.reset();
        return KYN_OK;
    }
    if (option == KYN_OPT_BULK_SECTIONS) {
        c->bulk_sections = value != 0;
        return KYN_OK;
    }
    if (option == KYN_OPT_RESET_SOLVE_STATS) {
        KYN_CUDA(c, cudaMemsetAsync(c->d_diag, 0, kNumDiag * sizeof(unsigned long long), c->stream));
        return KYN_OK;
    }
    if (option == KYN_OPT_LINEAR_SOLVER) {
        if (value != KYN_SOLVER_GAUSS_JORDAN && value != KYN_SOLVER_PANEL_LU)
            return set_err(c, KYN_ERR_INVALID, "unknown linear solver");
        if (c->solver != static_cast<int>(value)) c->plan.reset();  // buckets carry their solver
        c->solver = static_cast<int>(value);
        return KYN_OK;
    }
    if (option == KYN_OPT_CUDA_GRAPH) {
        c->use_graph = value != 0;
        c->plan.reset();
        return KYN_OK;
    }
    if (option == KYN_OPT_PHASE_TIMING) {
        KYN_CUDA(c, cudaStreamSynchronize(c->stream));
        if (value && !c->d_prof) {
            KYN_ALLOC(c, cudaMalloc(&c->d_prof, 16 * sizeof(unsigned long long)));
        }
        if (c->d_prof) KYN_CUDA(c, cudaMemset(c->d_prof, 0, 16 * sizeof(unsigned long long)));
        if (!value && c->d_prof) {
            cudaFree(c->d_prof);
            c->d_prof = nullptr;
        }
        c->plan.reset();
        return KYN_OK;
    }
    return set_err(c, KYN_ERR_INVALID, "unknown option");
}

int kyn_model_create(kyn_ctx* c, const kyn_model_desc* desc) {
    if (!c) return KYN_ERR_INVALID;
    cudaSetDevice(c->device);
    auto m = std::make_unique<DevModel>();
    std::string err;
    const int rc = build_host_model(desc, m->host, err);
    if (rc != KYN_OK) return set_err(c, rc, err);
    size_t bytes = kMaxNewtonIters * sizeof(double);
    for (auto& b : m->host.beams) {
        const int hubf = hub_kind(m->host);
        const int nt = b.dense ? 128 : beam_threads(b.N, b.Q, b.nc, sizeof(double), hubf);
        if (b.cond_nd > 0 && dense_smem(m->host, b, nt) > kMaxDynSmem) {
            // the condensed model's bordered system moves to device memory (the slab's tail)
            if (b.slab.size() & 1) b.slab.push_back(0.);
            b.cond_md_off = static_cast<int>(b.slab.size());
            b.slab.resize(b.slab.size() + static_cast<size_t>(b.cond_nd) * b.cond_nd, 0.);
        }
        const int sm = b.dense ? dense_smem(m->host, b, nt)
                               : std::max(beam_smem(b.N, b.Q, b.nc, sizeof(double), 512, hubf),
                                          beam_smem(b.N, b.Q, b.nc, sizeof(double), nt, hubf));
        if (sm > kMaxDynSmem)
            return set_err(c, KYN_ERR_UNSUPPORTED, "beam system does not fit in shared memory");
        m->nt.push_back(nt);
        bytes += b.slab.size() * sizeof(double);
    }
    if (c->budget && c->used + bytes > c->budget)
        return set_err(c, KYN_ERR_BUDGET, "HBM budget exceeded");
    for (auto& b : m->host.beams) {
        double* p = nullptr;
        KYN_ALLOC(c, cudaMallocAsync(&p, b.slab.size() * sizeof(double), c->stream));
        KYN_CUDA(c, cudaMemcpyAsync(p, b.slab.data(), b.slab.size() * sizeof(double),
                                    cudaMemcpyHostToDevice, c->stream));
        m->d_slab.push_back(p);
    }
    KYN_ALLOC(c, cudaMallocAsync(&m->d_conv, kMaxNewtonIters * sizeof(double), c->stream));
    KYN_CUDA(c, cudaMemsetAsync(m->d_conv, 0, kMaxNewtonIters * sizeof(double), c->stream));
    if (c->record) {
        size_t tot = 0;
        for (auto& b : m->host.beams) {
            const size_t nl = 6 * b.N + 6 * b.nc;
            m->dump_off.push_back(tot);
            tot += nl * nl + 2 * nl;
        }
        KYN_ALLOC(c, cudaMallocAsync(&m->d_dump, tot * sizeof(double), c->stream));
        KYN_CUDA(c, cudaMemsetAsync(m->d_dump, 0, tot * sizeof(double), c->stream));
    }
    // Stream-ordered: the uploads (from the model's own host copy, which it
    // keeps) complete before any later work on the context stream, so a step
    // in flight is not waited for.
    m->bytes = bytes;
    c->used += bytes;
    prepare_model(m.get());
    {
        const int urc = upload_templates(c, m.get());
        if (urc != KYN_OK) return urc;
    }
    const int id = c->next_id++;
    register_model(c, id, std::move(m));
    return id;
}

int kyn_model_destroy(kyn_ctx* c, int id) {
    if (!c) return KYN_ERR_INVALID;
    DevModel* m = find_model(c, id);
    if (!m) return set_err(c, KYN_ERR_NOT_FOUND, "unknown model id");
    // Stream-ordered frees: a step in flight that uses the model (its bucket
    // streams join the context stream) completes before the memory is reused.
    for (double* p : m->d_slab) KYN_CUDA(c, cudaFreeAsync(p, c->stream));
    if (m->d_conv) KYN_CUDA(c, cudaFreeAsync(m->d_conv, c->stream));
    if (m->d_dump) KYN_CUDA(c, cudaFreeAsync(m->d_dump, c->stream));
    if (m->d_kt) KYN_CUDA(c, cudaFreeAsync(m->d_kt, c->stream));
    c->used -= m->bytes;
    c->by_id[id] = nullptr;
    c->models.erase(id);
    // Cached plans, transfer plans and prescribed-motion targets built before
    // this call are not reused (each compares the count with the one it was
    // built at), so a cached list that held this id is never stepped again.
    ++c->destroy_epoch;
    return KYN_OK;
}

int kyn_model_info_get(kyn_ctx* c, int id, kyn_model_info* info) {
    if (!c || !info) return KYN_ERR_INVALID;
    DevModel* m = find_model(c, id);
    if (!m) return set_err(c, KYN_ERR_NOT_FOUND, "unknown model id");
    const bool lumped = !m->host.beams.empty() && m->host.beams[0].lumped;
    info->num_nodes = m->host.num_nodes;
    info->num_beams = lumped ? 0 : m->host.num_elements;
    info->num_constraints = m->host.num_constraints;
    info->num_system_dofs = m->host.nsys;
    info->num_dofs = m->host.ndofs;
    info->nnz = static_cast<int32_t>(m->host.col_inds.size());
    int mn = 0, mq = 0;
    for (auto& b : m->host.beams) {
        if (b.lumped) continue;
        mn = std::max(mn, b.N);
        mq = std::max(mq, b.Q);
    }
    info->max_beam_nodes = mn;
    info->max_beam_qps = mq;
    info->device_bytes = static_cast<int64_t>(m->bytes);
    info->condensed_dofs = m->host.beams.empty() ? 0 : m->host.beams[0].cond_nd;
    return KYN_OK;
}

int kyn_model_describe(const kyn_model_desc* desc, kyn_model_info* info, int32_t* row_ptrs,
                       int32_t* col_inds, char* err, int errlen) {
    if (!info) return KYN_ERR_INVALID;
    HostModel h;
    std::string msg;
    const int rc = build_host_model(desc, h, msg);
    if (rc != KYN_OK) {
        if (err && errlen > 0) std::snprintf(err, static_cast<size_t>(errlen), "%s", msg.c_str());
        return rc;
    }
    const bool lumped = !h.beams.empty() && h.beams[0].lumped;
    info->num_nodes = h.num_nodes;
    info->num_beams = lumped ? 0 : h.num_elements;
    info->num_constraints = h.num_constraints;
    info->num_system_dofs = h.nsys;
    info->num_dofs = h.ndofs;
    info->nnz = static_cast<int32_t>(h.col_inds.size());
    int mn = 0, mq = 0;
    int64_t bytes = kMaxNewtonIters * static_cast<int64_t>(sizeof(double));
    for (auto& b : h.beams) {
        bytes += static_cast<int64_t>(b.slab.size() * sizeof(double));
        if (b.lumped) continue;
        mn = std::max(mn, b.N);
        mq = std::max(mq, b.Q);
    }
    info->max_beam_nodes = mn;
    info->max_beam_qps = mq;
    info->device_bytes = bytes;
    info->condensed_dofs = h.beams.empty() ? 0 : h.beams[0].cond_nd;
    if (row_ptrs) std::copy(h.row_ptrs.begin(), h.row_ptrs.end(), row_ptrs);
    if (col_inds) std::copy(h.col_inds.begin(), h.col_inds.end(), col_inds);
    return KYN_OK;
}

int kyn_model_set_loads(kyn_ctx* c, int id, int which, const double* values) {
    if (!c || !values) return KYN_ERR_INVALID;
    DevModel* m = find_model(c, id);
    if (!m) return set_err(c, KYN_ERR_NOT_FOUND, "unknown model id");
    if (which != KYN_LOAD_NODE_FX && which != KYN_LOAD_STATE_F)
        return set_err(c, KYN_ERR_INVALID, "unknown load channel");
    if (which == KYN_LOAD_NODE_FX && m->host.beams[0].lumped)
        return set_err(c, KYN_ERR_UNSUPPORTED, "a model without beam elements has no node_FX");
    // Stage in pinned memory in beam-local order, then one copy per beam; node_FX
    // rows of the elements of a multi-element beam add up at shared nodes.
    size_t need = 0;
    for (auto& b : m->host.beams) need += 6 * b.N;
    if (c->h_stage_len < need) {
        if (c->h_stage) {
            KYN_CUDA(c, cudaStreamSynchronize(c->stream));
            cudaFreeHost(c->h_stage);
        }
        KYN_ALLOC(c, cudaMallocHost(&c->h_stage, need * sizeof(double)));
        c->h_stage_len = need;
    }
    KYN_CUDA(c, cudaStreamSynchronize(c->stream));
    size_t off = 0;
    for (size_t bi = 0; bi < m->host.beams.size(); ++bi) {
        const HostBeam& b = m->host.beams[bi];
        const SlabLayout L = make_slab_layout(b.N, b.Q);
        if (which == KYN_LOAD_NODE_FX && (b.elem_ids.size() > 1 || b.dense)) {
            for (int k = 0; k < 6 * b.N; ++k) c->h_stage[off + k] = 0.;
            for (size_t ei = 0; ei < b.elem_ids.size(); ++ei) {
                const int row = m->host.elem_row[b.elem_ids[ei]];
                const auto& loc = b.elem_local[ei];
                for (size_t k = 0; k < loc.size(); ++k)
                    for (int cc = 0; cc < 6; ++cc)
                        c->h_stage[off + loc[k] * 6 + cc] += values[(row + k) * 6 + cc];
            }
        } else {
            const size_t row = (which == KYN_LOAD_NODE_FX) ? m->host.elem_row[b.elem_ids[0]] : 0;
            for (int k = 0; k < b.N; ++k)
                for (int cc = 0; cc < 6; ++cc)
                    c->h_stage[off + k * 6 + cc] = (which == KYN_LOAD_NODE_FX)
                                                       ? values[(row + k) * 6 + cc]
                                                       : values[b.node_ids[k] * 6 + cc];
        }
        KYN_CUDA(c, cudaMemcpyAsync(m->d_slab[bi] + (which == KYN_LOAD_NODE_FX ? L.fx : L.f),
                                    c->h_stage + off, 6 * b.N * sizeof(double),
                                    cudaMemcpyHostToDevice, c->stream));
        off += 6 * b.N;
    }
    KYN_CUDA(c, cudaStreamSynchronize(c->stream));
    return KYN_OK;
}

int kyn_model_set_prescribed(kyn_ctx* c, int id, int cid, const double u[7]) {
    if (!c || !u) return KYN_ERR_INVALID;
    DevModel* m = find_model(c, id);
    if (!m) return set_err(c, KYN_ERR_NOT_FOUND, "unknown model id");
    if (cid < 0 || cid >= m->host.num_constraints)
        return set_err(c, KYN_ERR_INVALID, "constraint id out of range");
    if (cid == m->host.ah_con) return KYN_OK;  // a rigid joint reads no input
    if (cid == m->host.hub_con || cid == m->host.rev_con) {
        // the hub BC, or the revolute joint's torque: every beam keeps a copy
        const int r = cid == m->host.rev_con ? 1 : 0;
        for (size_t bi = 0; bi < m->host.beams.size(); ++bi) {
            const HostBeam& b = m->host.beams[bi];
            const SlabLayout L = make_slab_layout(b.N, b.Q);
            KYN_CUDA(c, cudaMemcpyAsync(m->d_slab[bi] + L.hub + r * kHubDoubles + hubrec::input, u,
                                        7 * sizeof(double), cudaMemcpyHostToDevice, c->stream));
        }
        KYN_CUDA(c, cudaStreamSynchronize(c->stream));
        return KYN_OK;
    }
    const int bi = m->host.con_beam[cid], slot = m->host.con_slot[cid];
    const HostBeam& b = m->host.beams[bi];
    const SlabLayout L = make_slab_layout(b.N, b.Q);
    KYN_CUDA(c, cudaMemcpyAsync(m->d_slab[bi] + L.con_input + slot * 7, u, 7 * sizeof(double),
                                cudaMemcpyHostToDevice, c->stream));
    KYN_CUDA(c, cudaStreamSynchronize(c->stream));
    return KYN_OK;
}

int kyn_step(kyn_ctx* c, const int* ids, int n, const kyn_step_params* p, int* status_out,
             int* iters_out) {
    int rc = kyn_step_async(c, ids, n, p);
    if (rc != KYN_OK) return rc;
    return kyn_step_wait(c, status_out, iters_out);
}

int kyn_step_async(kyn_ctx* c, const int* ids, int n, const kyn_step_params* p) {
    if (!c || !p || n < 0 || (n > 0 && !ids)) return KYN_ERR_INVALID;
    if (p->max_iter < 1 || !(p->h > 0.)) return set_err(c, KYN_ERR_INVALID, "bad step parameters");
    if (p->precision != KYN_PRECISION_FP64 && p->precision != KYN_PRECISION_FP32_REFINED)
        return set_err(c, KYN_ERR_INVALID, "unknown precision mode");
    cudaSetDevice(c->device);
    c->pending.assign(ids, ids + n);
    if (n == 0) return KYN_OK;
    Plan* plan = nullptr;
    int rc = get_plan(c, ids, n, p->precision, &plan);
    if (rc != KYN_OK) return rc;
    if (!c->use_graph) return launch_plan(c, plan, p);
    // CUDA graph: capture the step's launch sequence (fork, bucket kernels,
    // join, status copies) once per plan and coefficient set, then replay it.
    const StepCoeffs P = make_coeffs(c, p);
    if (!plan->graph || std::memcmp(&P, &plan->graph_coeffs, sizeof(P)) != 0) {
        rc = configure_smem(c);
        if (rc != KYN_OK) return rc;
        if (plan->graph) {
            KYN_CUDA(c, cudaGraphExecDestroy(plan->graph));
            plan->graph = nullptr;
        }
        KYN_CUDA(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        const int64_t before = c->launches;
        rc = launch_plan(c, plan, p);
        cudaGraph_t g = nullptr;
        const cudaError_t ce = cudaStreamEndCapture(c->stream, &g);
        c->launches = before;
        if (rc != KYN_OK) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        KYN_CUDA(c, ce);
        const cudaError_t ie = cudaGraphInstantiate(&plan->graph, g, 0);
        cudaGraphDestroy(g);
        KYN_CUDA(c, ie);
        plan->graph_coeffs = P;
    }
    KYN_CUDA(c, cudaGraphLaunch(plan->graph, c->stream));
    c->launches += static_cast<int64_t>(plan->buckets.size());
    c->last_buckets = static_cast<int64_t>(plan->buckets.size());
    return KYN_OK;
}

int kyn_step_wait(kyn_ctx* c, int* status_out, int* iters_out) {
    if (!c) return KYN_ERR_INVALID;
    if (c->pending.empty()) return KYN_OK;
    if (!c->plan) return set_err(c, KYN_ERR_INVALID, "no step in flight");
    return finish_plan(c, c->plan.get(), status_out, iters_out);
}

int kyn_get_state(kyn_ctx* c, int id, int field, double* out) {
    if (!c || !out) return KYN_ERR_INVALID;
    DevModel* m = find_model(c, id);
    if (!m) return set_err(c, KYN_ERR_NOT_FOUND, "unknown model id");
    KYN_CUDA(c, cudaStreamSynchronize(c->stream));
    const HostModel& HM = m->host;
    if (field == KYN_FIELD_CONSTRAINT_OUTPUT) {
        // Constraints::output (src/step/step.hpp:105-115): the revolute joint's
        // rotation, rate and acceleration about its axis
        // (src/constraints/calculate_revolute_joint_output.hpp:24-85), from beam
        // 0's copy of the azimuth record; zero for the other constraints.
        for (int k = 0; k < 3 * HM.num_constraints; ++k) out[k] = 0.;
        if (!HM.beams.empty() && HM.beams[0].dense && HM.beams[0].frames_off >= 0) {
            // dense models: every revolute joint, from its target node's state
            // in the one dense record and the joint frame kept in its slab
            const HostBeam& b0 = HM.beams[0];
            const SlabLayout L0 = make_slab_layout(b0.N, 0);
            for (int cid = 0; cid < HM.num_constraints; ++cid) {
                const int slot = HM.con_slot[cid];
                if (slot < 0 || b0.con_type[slot] != KYN_CONSTRAINT_REVOLUTE_JOINT) continue;
                const int n = b0.con_node[slot];
                double qv[7], w[6], wd[6];
                KYN_CUDA(c, cudaMemcpy(qv, m->d_slab[0] + L0.q + n * 7, sizeof(qv), cudaMemcpyDeviceToHost));
                KYN_CUDA(c, cudaMemcpy(w, m->d_slab[0] + L0.v + n * 6, sizeof(w), cudaMemcpyDeviceToHost));
                KYN_CUDA(c, cudaMemcpy(wd, m->d_slab[0] + L0.vd + n * 6, sizeof(wd), cudaMemcpyDeviceToHost));
                const double* q = qv + 3;
                const double* a0 = b0.slab.data() + b0.frames_off + slot * 9;
                double ax[3], rv[3] = {0., 0., 0.};
                for (int i = 0; i < 3; ++i) {
                    ax[i] = 0.;
                    for (int j = 0; j < 3; ++j) ax[i] += rot_entry(q, i, j) * a0[j];
                }
                const double sh = std::sqrt(1. - q[0] * q[0]);
                if (sh > 1e-12) {  // QuaternionToRotationVector (src/math/quaternion_operations.hpp:248-262)
                    const double th = 2. * std::acos(q[0]);
                    for (int i = 0; i < 3; ++i) rv[i] = th * q[1 + i] / sh;
                }
                double* o = out + 3 * cid;
                for (int i = 0; i < 3; ++i) {
                    o[0] += ax[i] * rv[i];
                    o[1] += ax[i] * w[3 + i];
                    o[2] += ax[i] * wd[3 + i];
                }
            }
            return KYN_OK;
        }
        if (HM.rev_con < 0) return KYN_OK;
        const HostBeam& b0 = HM.beams[0];
        const SlabLayout L0 = make_slab_layout(b0.N, b0.Q);
        double R[kHubDoubles];
        KYN_CUDA(c, cudaMemcpy(R, m->d_slab[0] + L0.hub + kHubDoubles, sizeof(R), cudaMemcpyDeviceToHost));
        const double* q = R + hubrec::q + 3;
        const double* a0 = R + hubrec::axes;
        double ax[3], rv[3] = {0., 0., 0.};
        for (int i = 0; i < 3; ++i) {
            ax[i] = 0.;
            for (int j = 0; j < 3; ++j) ax[i] += rot_entry(q, i, j) * a0[j];
        }
        const double sh = std::sqrt(1. - q[0] * q[0]);
        if (sh > 1e-12) {  // QuaternionToRotationVector (src/math/quaternion_operations.hpp:248-262)
            const double th = 2. * std::acos(q[0]);
            for (int i = 0; i < 3; ++i) rv[i] = th * q[1 + i] / sh;
        }
        double* o = out + 3 * HM.rev_con;
        for (int i = 0; i < 3; ++i) {
            o[0] += ax[i] * rv[i];
            o[1] += ax[i] * R[hubrec::v + 3 + i];
            o[2] += ax[i] * R[hubrec::vd + 3 + i];
        }
        return KYN_OK;
    }
    for (size_t bi = 0; bi < m->host.beams.size(); ++bi) {
        const HostBeam& b = m->host.beams[bi];
        const SlabLayout L = make_slab_layout(b.N, b.Q);
        std::vector<double> h(L.total);
        KYN_CUDA(c, cudaMemcpy(h.data(), m->d_slab[bi], L.total * sizeof(double),
                               cudaMemcpyDeviceToHost));
        if (field == KYN_FIELD_LAMBDA) {
            for (int s = 0; s < b.nc; ++s)
                for (int k = 0; k < 6; ++k) out[b.con_row[s] * 6 + k] = h[L.lambda + s * 6 + k];
            // the constraints leading into the hub-chain records: the hub BC, the
            // revolute joint, the rigid joint inside the drive train
            const int into[3] = {HM.hub_con, HM.rev_con, HM.ah_con};
            for (size_t r = 0; bi == 0 && r < HM.chain.size(); ++r)
                for (int k = 0; k < 6; ++k)
                    out[into[r] * 6 + k] = h[L.hub + r * kHubDoubles + hubrec::lambda + k];
            continue;
        }
        int src = -1, w = 0;
        switch (field) {
            case KYN_FIELD_X0: src = L.x0; w = 7; break;
            case KYN_FIELD_X: src = L.x; w = 7; break;
            case KYN_FIELD_Q: src = L.q; w = 7; break;
            case KYN_FIELD_Q_PREV: src = L.q_prev; w = 7; break;
            case KYN_FIELD_Q_DELTA: src = L.q_delta; w = 6; break;
            case KYN_FIELD_V: src = L.v; w = 6; break;
            case KYN_FIELD_VD: src = L.vd; w = 6; break;
            case KYN_FIELD_A: src = L.a; w = 6; break;
            case KYN_FIELD_F: src = L.f; w = 6; break;
            case KYN_FIELD_TANGENT: src = L.tangent; w = 36; break;
            default: return set_err(c, KYN_ERR_INVALID, "unknown state field");
        }
        for (int k = 0; k < b.N; ++k) {
            double* o = out + static_cast<size_t>(b.node_ids[k]) * w;
            if (field == KYN_FIELD_TANGENT) {
                for (int e = 0; e < 36; ++e) o[e] = 0.;
                for (int d = 0; d < 3; ++d) o[d * 7] = 1.;
                for (int i = 0; i < 3; ++i)
                    for (int j = 0; j < 3; ++j) o[(3 + i) * 6 + 3 + j] = h[src + k * 9 + i * 3 + j];
            } else {
                for (int e = 0; e < w; ++e) o[e] = h[src + k * w + e];
            }
        }
        for (size_t r = 0; bi == 0 && r < HM.chain.size(); ++r) {  // hub-chain nodes, from beam 0's copy
            const double* H = h.data() + L.hub + r * kHubDoubles;
            double* o = out + static_cast<size_t>(HM.chain[r]) * w;
            int hw = 0;
            const int ho = hub_field_offset(field, &hw);
            if (field == KYN_FIELD_TANGENT) {
                for (int e = 0; e < 36; ++e) o[e] = 0.;
                for (int d = 0; d < 3; ++d) o[d * 7] = 1.;
                for (int i = 0; i < 3; ++i)
                    for (int j = 0; j < 3; ++j) o[(3 + i) * 6 + 3 + j] = H[hubrec::tangent + i * 3 + j];
            } else if (ho >= 0) {
                for (int e = 0; e < w; ++e) o[e] = H[ho + e];
            } else {
                for (int e = 0; e < w; ++e) o[e] = 0.;
            }
        }
    }
    return KYN_OK;
}

int kyn_get_convergence(kyn_ctx* c, int id, double* errs, int* n) {
    if (!c) return KYN_ERR_INVALID;
    DevModel* m = find_model(c, id);
    if (!m) return set_err(c, KYN_ERR_NOT_FOUND, "unknown model id");
    KYN_CUDA(c, cudaStreamSynchronize(c->stream));
    const int cnt = std::min(m->last_iters, kMaxNewtonIters);
    if (errs && cnt > 0)
        KYN_CUDA(c, cudaMemcpy(errs, m->d_conv, cnt * sizeof(double), cudaMemcpyDeviceToHost));
    if (n) *n = cnt;
    return KYN_OK;
}

int kyn_get_crs(kyn_ctx* c, int id, int* row_ptrs, int* col_inds, double* values) {
    if (!c) return KYN_ERR_INVALID;
    DevModel* m = find_model(c, id);
    if (!m) return set_err(c, KYN_ERR_NOT_FOUND, "unknown model id");
    const HostModel& H = m->host;
    if (row_ptrs) std::copy(H.row_ptrs.begin(), H.row_ptrs.end(), row_ptrs);
    if (col_inds) std::copy(H.col_inds.begin(), H.col_inds.end(), col_inds);
    if (!values) return KYN_OK;
    if (m->host.hub >= 0 || m->host.beams[0].dense)
        return set_err(c, KYN_ERR_UNSUPPORTED,
                       "system values are not recorded for models with a hub or dense models");
    if (!m->d_dump) return set_err(c, KYN_ERR_INVALID, "KYN_OPT_RECORD_SYSTEM was not set");
    KYN_CUDA(c, cudaStreamSynchronize(c->stream));
    std::fill(values, values + H.col_inds.size(), 0.);
    for (size_t bi = 0; bi < H.beams.size(); ++bi) {
        const HostBeam& b = H.beams[bi];
        const int nl = 6 * b.N + 6 * b.nc;
        std::vector<double> D(static_cast<size_t>(nl) * nl);
        KYN_CUDA(c, cudaMemcpy(D.data(), m->d_dump + m->dump_off[bi], D.size() * sizeof(double),
                               cudaMemcpyDeviceToHost));
        auto gdof = [&](int l) {
            if (l < 6 * b.N) return H.fmap[b.node_ids[l / 6]] + l % 6;
            const int s = (l - 6 * b.N) / 6;
            return H.nsys + 6 * b.con_row[s] + (l - 6 * b.N) % 6;
        };
        for (int r = 0; r < nl; ++r) {
            const int gr = gdof(r);
            const int* beg = H.col_inds.data() + H.row_ptrs[gr];
            const int* end = H.col_inds.data() + H.row_ptrs[gr + 1];
            for (int cc = 0; cc < nl; ++cc) {
                const double v = D[static_cast<size_t>(r) * nl + cc];
                if (v == 0.) continue;
                const int gc = gdof(cc);
                const int* p = std::lower_bound(beg, end, gc);
                if (p != end && *p == gc) values[p - H.col_inds.data()] = v;
            }
        }
    }
    return KYN_OK;
}

int kyn_get_system_vectors(kyn_ctx* c, int id, double* rhs, double* solution) {
    if (!c) return KYN_ERR_INVALID;
    DevModel* m = find_model(c, id);
    if (!m) return set_err(c, KYN_ERR_NOT_FOUND, "unknown model id");
    if (m->host.hub >= 0 || m->host.beams[0].dense)
        return set_err(c, KYN_ERR_UNSUPPORTED,
                       "system values are not recorded for models with a hub or dense models");
    if (!m->d_dump) return set_err(c, KYN_ERR_INVALID, "KYN_OPT_RECORD_SYSTEM was not set");
    KYN_CUDA(c, cudaStreamSynchronize(c->stream));
    const HostModel& H = m->host;
    for (size_t bi = 0; bi < H.beams.size(); ++bi) {
        const HostBeam& b = H.beams[bi];
        const int nl = 6 * b.N + 6 * b.nc;
        std::vector<double> V(2 * nl);
        KYN_CUDA(c, cudaMemcpy(V.data(), m->d_dump + m->dump_off[bi] + static_cast<size_t>(nl) * nl,
                               V.size() * sizeof(double), cudaMemcpyDeviceToHost));
        for (int l = 0; l < nl; ++l) {
            int g;
            if (l < 6 * b.N) g = H.fmap[b.node_ids[l / 6]] + l % 6;
            else g = H.nsys + 6 * b.con_row[(l - 6 * b.N) / 6] + (l - 6 * b.N) % 6;
            if (rhs) rhs[g] = V[l];
            if (solution) solution[g] = V[nl + l];
        }
    }
    return KYN_OK;
}

int kyn_set_loads_batch(kyn_ctx* c, const int* ids, int n, int which, const double* values,
                        int on_device) {
    if (!c || n < 0 || (n > 0 && (!ids || !values))) return KYN_ERR_INVALID;
    if (which != KYN_LOAD_NODE_FX && which != KYN_LOAD_STATE_F)
        return set_err(c, KYN_ERR_INVALID, "unknown load channel");
    if (n == 0) return KYN_OK;
    cudaSetDevice(c->device);
    XferPlan* xp = nullptr;
    int rc = get_xfer(c, ids, n, which, &xp);
    if (rc != KYN_OK) return rc;
    const double* src = values;
    if (!on_device) {
        rc = ensure_stage(c, xp->total);
        if (rc != KYN_OK) return rc;
        KYN_CUDA(c, cudaMemcpyAsync(c->d_stage, values, sizeof(double) * xp->total,
                                    cudaMemcpyHostToDevice, c->stream));
        src = c->d_stage;
    }
    xfer_kernel<<<xp->nbeams, 128, 0, c->stream>>>(xp->d_beams, xp->d_map,
                                                   const_cast<double*>(src), 6, 1);
    KYN_CUDA(c, cudaGetLastError());
    c->launches++;
    return KYN_OK;
}

int kyn_get_state_batch(kyn_ctx* c, const int* ids, int n, int field, double* out, int on_device) {
    if (!c || n < 0 || (n > 0 && (!ids || !out))) return KYN_ERR_INVALID;
    if (n == 0) return KYN_OK;
    cudaSetDevice(c->device);
    XferPlan* xp = nullptr;
    int rc = get_xfer(c, ids, n, 100 + field, &xp);
    if (rc != KYN_OK) return rc;
    double* dst = out;
    if (!on_device) {
        rc = ensure_stage(c, xp->total);
        if (rc != KYN_OK) return rc;
        dst = c->d_stage;
    }
    xfer_kernel<<<xp->nbeams, 128, 0, c->stream>>>(xp->d_beams, xp->d_map, dst, xp->width, 0);
    KYN_CUDA(c, cudaGetLastError());
    c->launches++;
    if (!on_device) {
        KYN_CUDA(c, cudaMemcpyAsync(out, c->d_stage, sizeof(double) * xp->total,
                                    cudaMemcpyDeviceToHost, c->stream));
        KYN_CUDA(c, cudaStreamSynchronize(c->stream));
    }
    return KYN_OK;
}

}  // extern "C"

// ---- batched prescribed motion -------------------------------------------------
namespace {

// Target e (a constraint input slot, or one beam's copy of a hub BC input)
// receives the 7 values of row vidx[e] of the caller's array.
__global__ void prescribed_kernel(double* const* __restrict__ targets, const int* __restrict__ vidx,
                                  const double* __restrict__ vals, int count) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < count * 7) targets[t / 7][t % 7] = vals[vidx[t / 7] * 7 + t % 7];
}

}  // namespace

extern "C" int kyn_set_prescribed_batch(kyn_ctx* c, const int* ids, int n, const double* values,
                                        int on_device) {
    if (!c || n < 0 || (n > 0 && (!ids || !values))) return KYN_ERR_INVALID;
    if (n == 0) return KYN_OK;
    KYN_CUDA(c, cudaSetDevice(c->device));
    if (!(c->presc_epoch == c->destroy_epoch && static_cast<int>(c->presc_ids.size()) == n &&
          std::equal(ids, ids + n, c->presc_ids.begin()))) {
        std::vector<double*> t;
        std::vector<int> vi;
        int row = 0;
        for (int i = 0; i < n; ++i) {
            DevModel* m = find_model(c, ids[i]);
            if (!m) return set_err(c, KYN_ERR_NOT_FOUND, "unknown model id in batch");
            for (int k = 0; k < m->host.num_constraints; ++k, ++row) {
                if (k == m->host.ah_con) continue;  // a rigid joint reads no input
                if (k == m->host.hub_con || k == m->host.rev_con) {
                    const int r = k == m->host.rev_con ? 1 : 0;
                    for (size_t bi = 0; bi < m->host.beams.size(); ++bi) {
                        const HostBeam& b = m->host.beams[bi];
                        const SlabLayout L = make_slab_layout(b.N, b.Q);
                        t.push_back(m->d_slab[bi] + L.hub + r * kHubDoubles + hubrec::input);
                        vi.push_back(row);
                    }
                    continue;
                }
                const int bi = m->host.con_beam[k], slot = m->host.con_slot[k];
                const HostBeam& b = m->host.beams[bi];
                const SlabLayout L = make_slab_layout(b.N, b.Q);
                t.push_back(m->d_slab[bi] + L.con_input + slot * 7);
                vi.push_back(row);
            }
        }
        if (c->presc_cap < t.size() || !c->presc_targets) {
            size_t tcap = c->presc_cap, vcap = c->presc_cap;
            int rc = grow_device(c, c->presc_targets, tcap, t.size(), kPoolBeams);
            if (rc != KYN_OK) return rc;
            rc = grow_device(c, c->presc_vidx, vcap, t.size(), kPoolBeams);
            if (rc != KYN_OK) return rc;
            c->presc_cap = std::min(tcap, vcap);
        }
        if (!t.empty()) {
            KYN_CUDA(c, cudaMemcpyAsync(c->presc_targets, t.data(), sizeof(double*) * t.size(),
                                        cudaMemcpyHostToDevice, c->stream));
            KYN_CUDA(c, cudaMemcpyAsync(c->presc_vidx, vi.data(), sizeof(int) * vi.size(),
                                        cudaMemcpyHostToDevice, c->stream));
        }
        c->presc_count = static_cast<int>(t.size());
        c->presc_rows = row;
        c->presc_ids.assign(ids, ids + n);
        c->presc_epoch = c->destroy_epoch;
    }
    const int cnt = c->presc_count;
    if (cnt == 0) return KYN_OK;
    const double* src = values;
    if (!on_device) {
        int rc = ensure_stage(c, static_cast<long long>(c->presc_rows) * 7);
        if (rc != KYN_OK) return rc;
        KYN_CUDA(c, cudaMemcpyAsync(c->d_stage, values, sizeof(double) * 7 * c->presc_rows,
                                    cudaMemcpyHostToDevice, c->stream));
        src = c->d_stage;
    }
    prescribed_kernel<<<(cnt * 7 + 255) / 256, 256, 0, c->stream>>>(c->presc_targets, c->presc_vidx,
                                                                    src, cnt);
    KYN_CUDA(c, cudaGetLastError());
    c->launches++;
    return KYN_OK;
}

// ---- state save / restore / copy (restart files, predictor-corrector) -----------
namespace {

// Slab offset and row width of a node field.
int field_offset(int field, const SlabLayout& L, int* w) {
    switch (field) {
        case KYN_FIELD_X0: *w = 7; return L.x0;
        case KYN_FIELD_X: *w = 7; return L.x;
        case KYN_FIELD_Q: *w = 7; return L.q;
        case KYN_FIELD_Q_PREV: *w = 7; return L.q_prev;
        case KYN_FIELD_Q_DELTA: *w = 6; return L.q_delta;
        case KYN_FIELD_V: *w = 6; return L.v;
        case KYN_FIELD_VD: *w = 6; return L.vd;
        case KYN_FIELD_A: *w = 6; return L.a;
        case KYN_FIELD_F: *w = 6; return L.f;
        default: return -1;
    }
}

// Fields of the restart record, in file order (src/state/write_state_to_file.hpp:50-58).
constexpr int kRestartFields[9] = {KYN_FIELD_X0, KYN_FIELD_X, KYN_FIELD_Q_DELTA, KYN_FIELD_Q_PREV,
                                   KYN_FIELD_Q, KYN_FIELD_V, KYN_FIELD_VD, KYN_FIELD_A, KYN_FIELD_F};
constexpr int kRestartWidth[9] = {7, 7, 6, 7, 7, 6, 6, 6, 6};

}  // namespace

extern "C" int kyn_set_state(kyn_ctx* c, int id, int field, const double* values) {
    if (!c || !values) return KYN_ERR_INVALID;
    DevModel* m = find_model(c, id);
    if (!m) return set_err(c, KYN_ERR_NOT_FOUND, "unknown model id");
    KYN_CUDA(c, cudaStreamSynchronize(c->stream));
    for (size_t bi = 0; bi < m->host.beams.size(); ++bi) {
        const HostBeam& b = m->host.beams[bi];
        const SlabLayout L = make_slab_layout(b.N, b.Q);
        int w = 0;
        const int off = field_offset(field, L, &w);
        if (off < 0) return set_err(c, KYN_ERR_INVALID, "field cannot be set");
        std::vector<double> h(static_cast<size_t>(b.N) * w);
        for (int k = 0; k < b.N; ++k)
            for (int e = 0; e < w; ++e) h[k * w + e] = values[static_cast<size_t>(b.node_ids[k]) * w + e];
        KYN_CUDA(c, cudaMemcpy(m->d_slab[bi] + off, h.data(), h.size() * sizeof(double),
                               cudaMemcpyHostToDevice));
        int hw = 0;
        const int ho = hub_field_offset(field, &hw);
        for (size_t r = 0; ho >= 0 && r < m->host.chain.size(); ++r)  // every beam's copy of the hub chain
            KYN_CUDA(c, cudaMemcpy(m->d_slab[bi] + L.hub + r * kHubDoubles + ho,
                                   values + static_cast<size_t>(m->host.chain[r]) * w,
                                   w * sizeof(double), cudaMemcpyHostToDevice));
    }
    return KYN_OK;
}

extern "C" int kyn_state_write(kyn_ctx* c, int id, void* buf, size_t capacity, size_t* bytes) {
    if (!c || !bytes) return KYN_ERR_INVALID;
    DevModel* m = find_model(c, id);
    if (!m) return set_err(c, KYN_ERR_NOT_FOUND, "unknown model id");
    const size_t nn = static_cast<size_t>(m->host.num_nodes);
    size_t need = sizeof(size_t);
    for (int w : kRestartWidth) need += w * nn * sizeof(double);
    *bytes = need;
    if (!buf) return KYN_OK;
    if (capacity < need) return set_err(c, KYN_ERR_INVALID, "restart buffer too small");
    unsigned char* p = static_cast<unsigned char*>(buf);
    std::memcpy(p, &nn, sizeof(size_t));
    p += sizeof(size_t);
    std::vector<double> tmp(7 * nn);
    for (int f = 0; f < 9; ++f) {
        const int rc = kyn_get_state(c, id, kRestartFields[f], tmp.data());
        if (rc != KYN_OK) return rc;
        const size_t len = kRestartWidth[f] * nn * sizeof(double);
        std::memcpy(p, tmp.data(), len);
        p += len;
    }
    return KYN_OK;
}

extern "C" int kyn_state_read(kyn_ctx* c, int id, const void* buf, size_t size) {
    if (!c || !buf) return KYN_ERR_INVALID;
    DevModel* m = find_model(c, id);
    if (!m) return set_err(c, KYN_ERR_NOT_FOUND, "unknown model id");
    const size_t nn = static_cast<size_t>(m->host.num_nodes);
    if (size < sizeof(size_t)) return set_err(c, KYN_ERR_INVALID, "restart record too short");
    size_t file_nodes = 0;
    std::memcpy(&file_nodes, buf, sizeof(size_t));
    if (file_nodes != nn)
        return set_err(c, KYN_ERR_INVALID, "Number of system nodes in file is not the same as in model");
    size_t need = sizeof(size_t);
    for (int w : kRestartWidth) need += w * nn * sizeof(double);
    if (size < need) return set_err(c, KYN_ERR_INVALID, "restart record too short");
    const unsigned char* p = static_cast<const unsigned char*>(buf) + sizeof(size_t);
    std::vector<double> tmp(7 * nn);
    for (int f = 0; f < 9; ++f) {
        const size_t len = kRestartWidth[f] * nn * sizeof(double);
        std::memcpy(tmp.data(), p, len);
        p += len;
        const int rc = kyn_set_state(c, id, kRestartFields[f], tmp.data());
        if (rc != KYN_OK) return rc;
    }
    return KYN_OK;
}

extern "C" int kyn_state_copy(kyn_ctx* c, int dst, int src) {
    if (!c) return KYN_ERR_INVALID;
    DevModel* d = find_model(c, dst);
    DevModel* s = find_model(c, src);
    if (!d || !s) return set_err(c, KYN_ERR_NOT_FOUND, "unknown model id");
    if (d->host.beams.size() != s->host.beams.size() || d->host.chain.size() != s->host.chain.size())
        return set_err(c, KYN_ERR_INVALID, "models differ in structure");
    for (size_t bi = 0; bi < d->host.beams.size(); ++bi) {
        const HostBeam& a = d->host.beams[bi];
        const HostBeam& b = s->host.beams[bi];
        if (a.N != b.N || a.Q != b.Q || a.nc != b.nc)
            return set_err(c, KYN_ERR_INVALID, "models differ in structure");
    }
    // CopyStateData (src/state/copy_state_data.hpp:21-34): x, q_delta, q_prev, q, v,
    // vd, a, f, tangent -- the slab's state arrays from x through the tangent block
    for (size_t bi = 0; bi < d->host.beams.size(); ++bi) {
        const HostBeam& b = d->host.beams[bi];
        const SlabLayout L = make_slab_layout(b.N, b.Q);
        const int fields[] = {L.x, L.q, L.q_prev, L.q_delta, L.v, L.vd, L.a, L.f, L.tangent};
        const int widths[] = {7, 7, 7, 6, 6, 6, 6, 6, 9};
        for (int k = 0; k < 9; ++k)
            KYN_CUDA(c, cudaMemcpyAsync(d->d_slab[bi] + fields[k], s->d_slab[bi] + fields[k],
                                        sizeof(double) * widths[k] * b.N, cudaMemcpyDeviceToDevice,
                                        c->stream));
        for (size_t r = 0; r < d->host.chain.size(); ++r)  // hub-chain states (inputs stay the destination's)
            KYN_CUDA(c, cudaMemcpyAsync(d->d_slab[bi] + L.hub + r * kHubDoubles,
                                        s->d_slab[bi] + L.hub + r * kHubDoubles,
                                        sizeof(double) * hubrec::input, cudaMemcpyDeviceToDevice,
                                        c->stream));
    }
    return KYN_OK;
}

// ---- autotuner: threads per CTA per model size class -----------------------------
namespace {

// Copy of a model (description and current device state) for tuning runs.
int clone_model(kyn_ctx* c, int id) {
    DevModel* src = find_model(c, id);
    if (!src) return set_err(c, KYN_ERR_NOT_FOUND, "unknown model id");
    auto m = std::make_unique<DevModel>();
    m->host = src->host;
    m->nt = src->nt;
    size_t bytes = kMaxNewtonIters * sizeof(double);
    for (auto& b : m->host.beams) bytes += b.slab.size() * sizeof(double);
    if (c->budget && c->used + bytes > c->budget)
        return set_err(c, KYN_ERR_BUDGET, "HBM budget exceeded");
    for (size_t bi = 0; bi < m->host.beams.size(); ++bi) {
        double* p = nullptr;
        const size_t len = m->host.beams[bi].slab.size() * sizeof(double);
        KYN_ALLOC(c, cudaMallocAsync(&p, len, c->stream));
        KYN_CUDA(c, cudaMemcpyAsync(p, src->d_slab[bi], len, cudaMemcpyDeviceToDevice, c->stream));
        m->d_slab.push_back(p);
    }
    KYN_ALLOC(c, cudaMallocAsync(&m->d_conv, kMaxNewtonIters * sizeof(double), c->stream));
    KYN_CUDA(c, cudaMemcpyAsync(m->d_conv, src->d_conv, kMaxNewtonIters * sizeof(double),
                                cudaMemcpyDeviceToDevice, c->stream));
    if (src->d_dump) {  // the recorded-system buffer, when the source has one
        m->dump_off = src->dump_off;
        size_t tot = 0;
        for (size_t bi = 0; bi < m->host.beams.size(); ++bi) {
            const size_t nl = 6 * m->host.beams[bi].N + 6 * m->host.beams[bi].nc;
            tot += nl * nl + 2 * nl;
        }
        KYN_ALLOC(c, cudaMallocAsync(&m->d_dump, tot * sizeof(double), c->stream));
        KYN_CUDA(c, cudaMemsetAsync(m->d_dump, 0, tot * sizeof(double), c->stream));
    }
    m->last_status = src->last_status;
    m->last_iters = src->last_iters;
    m->bytes = bytes;
    c->used += bytes;
    prepare_model(m.get());
    {
        const int urc = upload_templates(c, m.get());
        if (urc != KYN_OK) return urc;
    }
    const int nid = c->next_id++;
    register_model(c, nid, std::move(m));
    return nid;
}

}  // namespace

extern "C" int kyn_model_clone(kyn_ctx* c, int model_id) {
    if (!c) return KYN_ERR_INVALID;
    KYN_CUDA(c, cudaSetDevice(c->device));
    return clone_model(c, model_id);
}

extern "C" int kyn_autotune(kyn_ctx* c, const int* ids, int n, const kyn_step_params* p) {
    if (!c || !p || n < 0 || (n > 0 && !ids)) return KYN_ERR_INVALID;
    if (p->precision != KYN_PRECISION_FP64 && p->precision != KYN_PRECISION_FP32_REFINED)
        return set_err(c, KYN_ERR_INVALID, "unknown precision mode");
    if (n == 0) return KYN_OK;
    KYN_CUDA(c, cudaSetDevice(c->device));
    const int rb = (p->precision == KYN_PRECISION_FP32_REFINED) ? 4 : 8;
    int sms = 148;
    KYN_CUDA(c, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device));
    const size_t sample_max = 16384;  // copies timed per class at most
    std::map<ClassKey, std::vector<int>> classes;
    for (int i = 0; i < n; ++i) {
        DevModel* m = find_model(c, ids[i]);
        if (!m) return set_err(c, KYN_ERR_NOT_FOUND, "unknown model id in autotune list");
        classes[class_key(m->host, p->precision)].push_back(ids[i]);
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    KYN_CUDA(c, cudaEventCreate(&e0));
    KYN_CUDA(c, cudaEventCreate(&e1));
    int rc = KYN_OK;
    for (auto& kv : classes) {
        const ClassKey& key = kv.first;
        // copies of all the class's models (the batch being tuned), repeated up
        // to 4 x SMs so that a small class is timed on full waves of CTAs
        std::vector<int> clones;
        const size_t nsrc = kv.second.size();
        const size_t want = std::min(std::max(nsrc, static_cast<size_t>(4) * sms), sample_max);
        for (size_t j = 0; j < want; ++j) {
            const int cid = clone_model(c, kv.second[j % nsrc]);
            if (cid < 0) break;
            clones.push_back(cid);
        }
        if (clones.empty()) continue;
        const HostModel& h = find_model(c, clones[0])->host;
        const int def_nt = find_model(c, clones[0])->def_nt[rb == 4 ? 1 : 0];
        // Every candidate is timed on the same two steps from the sources'
        // current state (the clones are reset before the warm-up and before the
        // timed steps), so that Newton iteration counts match across candidates.
        auto reset = [&]() {
            for (size_t j = 0; j < clones.size(); ++j) {
                const int r2 = kyn_state_copy(c, clones[j], kv.second[j % nsrc]);
                if (r2 != KYN_OK) return r2;
            }
            return static_cast<int>(KYN_OK);
        };
        // candidates: threads per CTA, and in the FP64 form for plain beam
        // systems also the free-block solver (panel LU or register
        // Gauss-Jordan: the same FP64 accuracy class, different speeds by size)
        const bool try_solver = p->precision == KYN_PRECISION_FP64 && find_model(c, clones[0])->lump == 0;
        const int other = c->solver == KYN_SOLVER_PANEL_LU ? KYN_SOLVER_GAUSS_JORDAN : KYN_SOLVER_PANEL_LU;
        int best_nt = -1, best_sv = c->solver;
        float best_ms = 0.f, def_ms = -1.f;
        for (int nt : {128, 256, 512}) {
            bool fits = true;
            for (const HostBeam& b : h.beams)
                fits &= (b.dense ? dense_smem(h, b, nt)
                                 : beam_smem(b.N, b.Q, b.nc, rb, nt, hub_kind(h))) <= kMaxDynSmem;
            if (!fits || (key.beams > 1 && key.beams * nt > 1024 * 8)) continue;
            for (int sv : {c->solver, other}) {
                if (sv != c->solver && !try_solver) continue;
                c->tuned[key] = nt;
                c->tuned_solver[key] = sv;
                ++c->tuned_gen;
                c->plan.reset();
                Plan* plan = nullptr;
                rc = get_plan(c, clones.data(), static_cast<int>(clones.size()), p->precision, &plan);
                if (rc == KYN_OK) rc = reset();
                if (rc == KYN_OK) rc = launch_plan(c, plan, p);  // warm-up step
                if (rc == KYN_OK) rc = finish_plan(c, plan, nullptr, nullptr);
                if (rc == KYN_OK) rc = reset();
                if (rc != KYN_OK) break;
                KYN_CUDA(c, cudaEventRecord(e0, c->stream));
                for (int r = 0; r < 4 && rc == KYN_OK; ++r) rc = launch_plan(c, plan, p);
                KYN_CUDA(c, cudaEventRecord(e1, c->stream));
                if (rc == KYN_OK) rc = finish_plan(c, plan, nullptr, nullptr);
                if (rc != KYN_OK) break;
                float ms = 0.f;
                KYN_CUDA(c, cudaEventElapsedTime(&ms, e0, e1));
                if (nt == def_nt && sv == c->solver) def_ms = ms;
                if (best_nt < 0 || ms < best_ms) {
                    best_nt = nt;
                    best_sv = sv;
                    best_ms = ms;
                }
            }
            if (rc != KYN_OK) break;
        }
        // keep the default unless another choice is clearly faster (timing noise)
        if (def_ms > 0.f && (best_nt != def_nt || best_sv != c->solver) && best_ms > 0.97f * def_ms) {
            best_nt = def_nt;
            best_sv = c->solver;
        }
        if (best_nt > 0) {
            c->tuned[key] = best_nt;
            c->tuned_solver[key] = best_sv;
        } else {
            c->tuned.erase(key);
            c->tuned_solver.erase(key);
        }
        ++c->tuned_gen;
        c->plan.reset();
        for (int cid : clones) kyn_model_destroy(c, cid);
        if (rc != KYN_OK) break;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    c->plan.reset();
    return rc;
}

extern "C" int kyn_tuned_threads(kyn_ctx* c, int model_id, int precision) {
    if (!c) return KYN_ERR_INVALID;
    DevModel* m = find_model(c, model_id);
    if (!m) return set_err(c, KYN_ERR_NOT_FOUND, "unknown model id");
    const auto it = c->tuned.find(class_key(m->host, precision));
    if (it != c->tuned.end()) return it->second;
    const int rb = (precision == KYN_PRECISION_FP32_REFINED) ? 4 : 8;
    int nt = 128;
    for (const HostBeam& b : m->host.beams) nt = std::max(nt, beam_threads(b.N, b.Q, b.nc, rb, hub_kind(m->host)));
    return nt;
}

extern "C" int kyn_tuned_solver(kyn_ctx* c, int model_id, int precision) {
    if (!c) return KYN_ERR_INVALID;
    DevModel* m = find_model(c, model_id);
    if (!m) return set_err(c, KYN_ERR_NOT_FOUND, "unknown model id");
    const auto it = c->tuned_solver.find(class_key(m->host, precision));
    return it != c->tuned_solver.end() ? it->second : c->solver;
}

// ---- batched load scatter through a static staging array (no allocation) ----
//
// kyn_set_loads_batch stages host loads in a device buffer that the context
// grows with cudaMalloc, and builds its per-beam copy plan in cudaMalloc'd
// memory.  Some callers cannot let a library allocate while they run: a CFD
// solver that couples to the beams usually owns the device memory through its
// own pool and shares the GPU with this library, and cudaMalloc/cudaFree there
// would fail for lack of memory or stall the solver's streams with an implicit
// device synchronisation.  kyn_set_loads_batch_static does the same scatter
// (same kernel, same results) with every byte it needs on the device taken from
// one file-scope array of fixed size, and its host-side plan built in fixed
// static host arrays, so a call allocates nothing.
namespace {

constexpr int kStaticStageBeams = 8192;          // beam elements per call
constexpr int kStaticStageRows = 8192 * 32;      // node rows per call (8192 beams x 32 nodes)
constexpr long long kStaticStageValues = 1LL << 20;  // load doubles per call (8 MiB)
constexpr size_t kStaticBeamBytes = sizeof(XferBeam) * kStaticStageBeams;
constexpr size_t kStaticMapBytes = sizeof(int) * kStaticStageRows;
constexpr size_t kStaticValuesOffset = kStaticBeamBytes + kStaticMapBytes;
constexpr size_t kStaticStageBytes = kStaticValuesOffset + sizeof(double) * kStaticStageValues;
static_assert(kStaticBeamBytes % 256 == 0 && kStaticValuesOffset % 256 == 0,
              "static staging regions must stay 256-byte aligned");

// [copy plan: XferBeam x 8192 | node map: int x 262144 | load values: double x 2^20],
// 9.19 MiB in all.  Shared by every call on a device (and by every context on
// it); each call writes the part it reads before its kernel runs, so nothing
// has to start at zero and stale contents of an earlier call are never read.
static __device__ __align__(256) unsigned char g_static_stage[kStaticStageBytes];

constexpr int kStaticMaxDevices = 64;
std::mutex g_static_stage_mu;                        // guards the tables below
unsigned char* g_static_stage_addr[kStaticMaxDevices] = {};
XferBeam g_static_host_beams[kStaticStageBeams];     // host side of the copy plan
int g_static_host_map[kStaticStageRows];

// Set-up, once per device with that device current: the device address of
// g_static_stage.  Runs inside the first call on each device.
int static_stage_address(kyn_ctx* c, unsigned char** out) {
    if (c->device < 0 || c->device >= kStaticMaxDevices)
        return set_err(c, KYN_ERR_UNSUPPORTED, "static staging supports device ordinals below 64");
    if (!g_static_stage_addr[c->device]) {
        unsigned char* ptr = nullptr;
        const cudaError_t e = cudaGetSymbolAddress((void**)&ptr, g_static_stage);
        if (e != cudaSuccess || !ptr)
            return set_err(c, KYN_ERR_CUDA,
                           std::string("cudaGetSymbolAddress(static staging): ") + cudaGetErrorString(e));
        g_static_stage_addr[c->device] = ptr;
    }
    *out = g_static_stage_addr[c->device];
    return KYN_OK;
}

}  // namespace

extern "C" {

int kyn_set_loads_batch_static(kyn_ctx* c, const int* ids, int n, int which,
                               const double* values, int on_device) {
    if (!c || n < 0 || (n > 0 && (!ids || !values))) return KYN_ERR_INVALID;
    if (which != KYN_LOAD_NODE_FX && which != KYN_LOAD_STATE_F)
        return set_err(c, KYN_ERR_INVALID, "unknown load channel");
    if (n == 0) return KYN_OK;
    KYN_CUDA(c, cudaSetDevice(c->device));
    std::lock_guard<std::mutex> lock(g_static_stage_mu);
    unsigned char* base = nullptr;
    int rc = static_stage_address(c, &base);
    if (rc != KYN_OK) return rc;

    // Copy plan on the host (same rows and offsets as kyn_set_loads_batch).
    int nb = 0, rows = 0;
    long long off = 0;
    for (int i = 0; i < n; ++i) {
        DevModel* m = find_model(c, ids[i]);
        if (!m) return set_err(c, KYN_ERR_NOT_FOUND, "unknown model id in batch");
        long long elem = 0;
        for (size_t bi = 0; bi < m->host.beams.size(); ++bi) {
            const HostBeam& b = m->host.beams[bi];
            if (nb == kStaticStageBeams)
                return set_err(c, KYN_ERR_INVALID,
                               "kyn_set_loads_batch_static: more than 8192 beam elements in one call");
            if (rows + b.N > kStaticStageRows)
                return set_err(c, KYN_ERR_INVALID,
                               "kyn_set_loads_batch_static: more than 262144 node rows in one call");
            const SlabLayout L = make_slab_layout(b.N, b.Q);
            XferBeam xb{};
            xb.N = b.N;
            xb.map_off = rows;
            if (which == KYN_LOAD_NODE_FX) {
                if (b.elem_ids.size() != 1 || b.dense)
                    return set_err(c, KYN_ERR_UNSUPPORTED,
                                   "batched node_FX needs single-element beams (use kyn_model_set_loads)");
                xb.slab_field = m->d_slab[bi] + L.fx;
                xb.ext_off = off + elem * 6;
                for (int k = 0; k < b.N; ++k) g_static_host_map[rows + k] = k;
            } else {
                xb.slab_field = m->d_slab[bi] + L.f;
                xb.ext_off = off;
                for (int k = 0; k < b.N; ++k) g_static_host_map[rows + k] = b.node_ids[k];
            }
            g_static_host_beams[nb++] = xb;
            rows += b.N;
            elem += b.N;
        }
        off += (which == KYN_LOAD_NODE_FX) ? elem * 6 : static_cast<long long>(m->host.num_nodes) * 6;
    }
    if (!on_device && off > kStaticStageValues)
        return set_err(c, KYN_ERR_INVALID,
                       "kyn_set_loads_batch_static: " + std::to_string(off) +
                           " load values exceed the static staging maximum of 1048576 doubles");
    if (nb == 0) return KYN_OK;

    // Pageable host arrays: each copy returns once the driver holds the data,
    // so the next call may refill them.
    XferBeam* d_beams = reinterpret_cast<XferBeam*>(base);
    int* d_map = reinterpret_cast<int*>(base + kStaticBeamBytes);
    KYN_CUDA(c, cudaMemcpyAsync(d_beams, g_static_host_beams, sizeof(XferBeam) * nb,
                                cudaMemcpyHostToDevice, c->stream));
    KYN_CUDA(c, cudaMemcpyAsync(d_map, g_static_host_map, sizeof(int) * rows,
                                cudaMemcpyHostToDevice, c->stream));
    const double* src = values;
    if (!on_device) {
        double* d_values = reinterpret_cast<double*>(base + kStaticValuesOffset);
        KYN_CUDA(c, cudaMemcpyAsync(d_values, values, sizeof(double) * off,
                                    cudaMemcpyHostToDevice, c->stream));
        src = d_values;
    }
    xfer_kernel<<<nb, 128, 0, c->stream>>>(d_beams, d_map, const_cast<double*>(src), 6, 1);
    KYN_CUDA(c, cudaGetLastError());
    c->launches++;
    return KYN_OK;
}

}  // extern "C"
