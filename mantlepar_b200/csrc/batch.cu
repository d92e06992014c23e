// Batched transport: many independent meshes of uneven size advanced
// together, each with its own dt, CFL retries, balance check and status.
//
// Every stage is one launch per kernel over ALL active instances: a device
// work map sends each thread block to (instance, tile) and the block's
// instance record holds that instance's buffers and tables. The per-element
// arithmetic is the single-instance path's (stage_kernels.cuh; for general
// quad meshes quad_kernels.cuh, over the quad instances' own work lists), and
// the block grouping of the reductions is per instance, so each instance's
// result is bitwise the same alone and in a batch.
//
// The step logic is the reference's Run loop (src/couple/evolve.cpp:449-507)
// applied per instance: dt = min(cap, cfl/rate), stage-1 admissibility,
// courant check over the stage rates, admissibility of the combined state,
// halve-and-retry (<= 40), balance check, rollback on failure. Instances that
// need a retry run the next attempt while finished instances wait.
#include "common.hpp"
#include "phase_math.cuh"
#include "stage_device.cuh"
#include "stage_kernels.cuh"
#include "step_ctl.cuh"
#include "tables.hpp"
#include "quad_kernels.cuh"
#include "quad_tables.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

namespace mp {

PhaseConst phase_const(const mp_material& p, const mp_derived& d);
mp_status derive_checked(const mp_material& p, mp_derived& d);
mp_status validate_opts(const mp_transport_opts& o, mp_derived* der_out);

namespace {


// Stage kinds: P evaluates L(U^n) (store L), B the second stage (RK combine
// into S2), C the third stage of SSPRK3 (RK combine into S1).
enum : int { KIND_P = 0, KIND_B = 1, KIND_C = 2, NKIND = 3 };

// Per-instance records of one stage kind, read by the batched kernels.
template <class R>
struct InstArgs {
    ReconArgs<R> recon;
    CellPhaseArgs<R> phase;
    FaceArgs<R> face;
    SumArgs sum;
};

struct AxpyArgs {
    int n;
    const double *H0, *C0, *LH, *LC;
    double *H1, *C1;
    const double* dtp;
    double area;
    Partial* partial;
    const double* cell_area;   // per-cell areas (general quad mesh), else null
};

// Commit of an accepted step: the stage state that holds U^{n+1} becomes U^n.
struct CommitArgs {
    int n;
    const double *srcH, *srcC;
    double *dstH, *dstC;
};

// Work items: block -> instance and the first element of its tile (faces:
// edges [a, b); reconstruction: columns from a, row b).
struct Work { int inst, a, b, part; };

struct Tuning { int bx = 32, by = 4, cpt = 1; };

// ------------------------------------------------------------ batched kernels

template <class R>
__global__ void __launch_bounds__(128) batch_recon_kernel(const InstArgs<R>* args, const Work* work, const int* active,
                                                          Physics ph, int cpt) {
    const Work w = work[blockIdx.x];
    if (!active[w.inst]) return;
    const ReconArgs<R>& a = args[w.inst].recon;
    const int j = w.b + threadIdx.y;
    for (int c = 0; c < cpt; ++c) recon_cell(a, ph, w.a + c * blockDim.x + threadIdx.x, j);
}

// kExt: the adiabatic source (alpha0 != 0) is compiled in.
template <class R, bool kExt>
__global__ void __launch_bounds__(128, 8) batch_phase_kernel(const InstArgs<R>* args, const Work* work, const int* active,
                                                          Physics ph) {
    const Work w = work[blockIdx.x];
    if (!active[w.inst]) return;
    cellphase_cell<R, kExt>(args[w.inst].phase, ph, (long long)w.a + threadIdx.x);
}

template <class R>
__global__ void __launch_bounds__(128, 5) batch_face_kernel(const InstArgs<R>* args, const Work* work, const int* active,
                                                         Physics ph) {
    const Work w = work[blockIdx.x];
    if (!active[w.inst]) return;
    const long long e = (long long)w.a + threadIdx.x;
    if (e < w.b) face_edge(args[w.inst].face, ph, e);
}

template <class R>
__global__ void __launch_bounds__(128) batch_diffusion_kernel(const InstArgs<R>* args, const Work* work, const int* active,
                                                              Physics ph) {
    const Work w = work[blockIdx.x];
    if (!active[w.inst]) return;
    const long long e = (long long)w.a + threadIdx.x;
    if (e < w.b) diffusion_edge(args[w.inst].face, ph, e);
}

// General quad meshes: the per-element bodies of the single-mesh quad
// kernels (quad_kernels.cuh) over the quad instances' work lists.
__global__ void __launch_bounds__(128, 3) batch_quad_weno_kernel(const QuadStageArgs* args, const Work* work,
                                                                 const int* active) {
    const Work w = work[blockIdx.x];
    if (!active[w.inst]) return;
    const QuadStageArgs& a = args[w.inst];
    const int i = w.a + threadIdx.x, j = w.b + threadIdx.y;
    if (i < a.nx && j < a.ny) quad_weno_cell(a, i, j);
}

__global__ void __launch_bounds__(128, 4) batch_quad_limit_kernel(const QuadStageArgs* args, const Work* work,
                                                                  const int* active, Physics ph) {
    const Work w = work[blockIdx.x];
    if (!active[w.inst]) return;
    const QuadStageArgs& a = args[w.inst];
    const int i = w.a + threadIdx.x, j = w.b + threadIdx.y;
    if (i < a.nx && j < a.ny) quad_limit_cell(a, ph, i, j);
}

__global__ void __launch_bounds__(128, 4) batch_quad_phase_kernel(const QuadStageArgs* args, const Work* work,
                                                                  const int* active, Physics ph) {
    const Work w = work[blockIdx.x];
    if (!active[w.inst]) return;
    const QuadStageArgs& a = args[w.inst];
    const long long cell = (long long)w.a + threadIdx.x;
    if (cell < (long long)a.nx * a.ny) quad_cellphase_cell(a, ph, cell);
}

__global__ void __launch_bounds__(128, 4) batch_quad_face_kernel(const QuadStageArgs* args, const Work* work,
                                                                 const int* active, Physics ph) {
    const Work w = work[blockIdx.x];
    if (!active[w.inst]) return;
    const long long e = (long long)w.a + threadIdx.x;
    if (e < w.b) quad_face_edge(args[w.inst], ph, e);
}

__global__ void __launch_bounds__(128) batch_quad_diffusion_kernel(const QuadStageArgs* args, const Work* work,
                                                                   const int* active, Physics ph) {
    const Work w = work[blockIdx.x];
    if (!active[w.inst]) return;
    const long long e = (long long)w.a + threadIdx.x;
    if (e < w.b) quad_diffusion_edge(args[w.inst], ph, e);
}

// kSrc: the adiabatic source terms are added. An instance with per-cell
// areas (a general quad mesh) takes them.
template <class R, bool kSrc>
__global__ void __launch_bounds__(kRedBlock) batch_sum_kernel(const InstArgs<R>* args, const Work* work, const int* active) {
    const Work w = work[blockIdx.x];
    if (!active[w.inst]) return;
    const SumArgs& a = args[w.inst].sum;
    const Partial v = a.cell_area ? sum_cells<kSrc, true>(a, w.a) : sum_cells<kSrc>(a, w.a);
    block_reduce_write(v, a.partial + w.part);
}

__global__ void __launch_bounds__(kRedBlock) batch_axpy_kernel(const AxpyArgs* args, const Work* work, const int* active) {
    const Work w = work[blockIdx.x];
    if (!active[w.inst]) return;
    const AxpyArgs& a = args[w.inst];
    const Partial v = axpy_cells(a.n, a.H0, a.C0, a.LH, a.LC, *a.dtp, a.area, a.H1, a.C1, w.a, a.cell_area);
    block_reduce_write(v, a.partial + w.part);
}

// Copy of U^{n+1} into U^n for the instances that accepted their step (the
// accumulation work list: kSumCells cells per block).
__global__ void __launch_bounds__(kRedBlock) batch_commit_kernel(const CommitArgs* args, const Work* work,
                                                                 const int* active) {
    const Work w = work[blockIdx.x];
    if (!active[w.inst]) return;
    const CommitArgs& a = args[w.inst];
#pragma unroll
    for (int q = 0; q < kSumPer; ++q) {
        const long long k = (long long)w.a + q * kRedBlock + threadIdx.x;
        if (k < a.n) { a.dstH[k] = a.srcH[k]; a.dstC[k] = a.srcC[k]; }
    }
}

// One block per instance: fixed-order reduction of its block partials (the
// same thread/tree shape as the single-instance reduction, so totals agree
// bit for bit).
__global__ void __launch_bounds__(1024) batch_reduce_kernel(const Partial* partial, const int* part_off,
                                                           const int* part_cnt, const int* active, Totals* out) {
    const int inst = blockIdx.x;
    if (!active[inst]) return;
    const int off = part_off[inst], cnt = part_cnt[inst];
    Partial v = partial_identity();
    for (int b = threadIdx.x; b < cnt; b += blockDim.x) fold_partial(v, partial[off + b]);
    __shared__ Partial result;
    block_reduce_write(v, &result);
    __syncthreads();
    if (threadIdx.x == 0)
        out[inst] = Totals{result.maxRate, result.divergence, result.bH, result.bC, result.HI, result.CI,
                           result.Hmin, result.Cmin, result.Cmax, result.nonfinite, result.sH};
}

}  // namespace
}  // namespace mp

// ----------------------------------------------------------------- instance

struct MPInstance {
    bool used = false;
    mp_mesh_desc mesh{};
    int nx = 0, ny = 0;
    size_t N = 0, NE = 0, bytes = 0;
    void* arena = nullptr;            // one allocation per instance
    double *H, *C, *S1H, *S1C, *S2H, *S2C, *LH, *LC, *T, *phi, *rec, *rate, *vsn, *udn, *face;
    unsigned char* flags;
    mp::StageTables* tab;
    mp::StageTables host_tab;
    // Adiabatic source (alpha0 != 0): vertical solid and Darcy velocities at
    // the 25 cell quadrature points and the per-cell source sums, one
    // allocation made by mp_batch_set_cell_velocity.
    void* src_arena = nullptr;
    size_t src_bytes = 0;
    double *cvs_y = nullptr, *cud_y = nullptr, *srcH = nullptr, *srcR = nullptr, *srcS = nullptr;
    // General quad mesh (mp_batch_add_quads): per-cell tables, vertices and
    // edge spacing in one allocation, and the cell areas inside it.
    bool quad = false;
    double* qbuf = nullptr;
    size_t qbytes = 0;
    mp::QuadDev qdev{};
    const double* cell_area = nullptr;
    double time = 0.0;
    double t_end = INFINITY;          // time.end of this instance
    int accepted = 0;
    bool have_L = false;
    mp::Totals cur{};
    int status = 0;                   // sticky failure status
};

// time.end reached (src/couple/evolve.cpp:450-451: within 32 eps of the end).
static bool finished(const MPInstance& in) {
    if (!std::isfinite(in.t_end)) return false;
    const double remaining = in.t_end - in.time;
    return remaining <= 32 * 2.220446049250313e-16 * std::max(1.0, std::fabs(in.t_end));
}

struct mp_batch {
    mp_transport_opts opts;
    mp_derived der;
    mp::Physics ph;
    cudaStream_t stream = nullptr;
    std::vector<MPInstance> inst;
    // device tables rebuilt when the set changes
    bool dirty = true;
    int slots = 0;                     // capacity of the per-instance device arrays
    void* d_args[mp::NKIND] = {nullptr, nullptr, nullptr};
    mp::AxpyArgs* d_axpy = nullptr;
    mp::Work *d_wrecon = nullptr, *d_wphase = nullptr, *d_wface = nullptr, *d_wsum = nullptr;
    // Work lists: filled entries n_w*, allocated (and launched) cap_w*; the
    // entries past n_w* name the sentinel slot `slots`, never active, so a
    // change of the instance set rewrites contents only and the captured
    // graph stays valid until a capacity grows.
    int n_wrecon = 0, n_wphase = 0, n_wface = 0, n_wsum = 0;
    int cap_wrecon = 0, cap_wphase = 0, cap_wface = 0, cap_wsum = 0;
    // General quad meshes: their own stage records and work lists (the
    // accumulation, axpy and commit lists cover every instance).
    bool has_quads = false;            // launch the quad kernels (set by the first quad instance)
    void* d_qargs[mp::NKIND] = {nullptr, nullptr, nullptr};
    mp::Work *d_wqrec = nullptr, *d_wqphase = nullptr, *d_wqface = nullptr;
    int n_wqrec = 0, n_wqphase = 0, n_wqface = 0;
    int cap_wqrec = 0, cap_wqphase = 0, cap_wqface = 0;
    int *d_active = nullptr, *d_part_off = nullptr, *d_part_cnt = nullptr;
    mp::Partial* d_partial = nullptr;
    int partial_cap = 0;
    mp::Totals* d_tot = nullptr;
    mp::Totals* h_tot = nullptr;
    unsigned long long* d_status = nullptr;
    unsigned long long* h_status = nullptr;
    double* d_dt = nullptr;
    double* h_dt = nullptr;
    int* h_active = nullptr;
    mp::Tuning tune;
    size_t bytes_in_use = 0;
    // Device-resident stepping: one CUDA graph runs up to kGraphChunk steps
    // of every instance (step and attempt loops as conditional WHILE nodes,
    // decisions by the step controller); rebuilt when captured arguments
    // change (gen).
    bool use_graph = true;
    unsigned long long gen = 1, graph_gen = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    int graph_slots = 0;
    mp::InstCtl *d_ctl = nullptr, *h_ctl = nullptr;
    mp::CtlHeader *d_hdr = nullptr, *h_hdr = nullptr;
    mp_step_report *d_rep = nullptr, *h_rep = nullptr;
    mp::CommitArgs* d_commit = nullptr;
    int stage_kernels = 0;             // kernels of one stage kind (graph launch count)
    unsigned long long host_syncs = 0; // host waits of the stepping calls
    unsigned long long captures = 0;   // graph captures
    // profiling
    bool profile = false;
    std::vector<cudaEvent_t> ev_pool;
    std::vector<int> ev_kind;
    size_t ev_used = 0;
    double kern_ms[6] = {0, 0, 0, 0, 0, 0};
    unsigned long long kern_n[6] = {0, 0, 0, 0, 0, 0};
};

namespace mp {
namespace {

size_t align256(size_t b) { return (b + 255) / 256 * 256; }

size_t instance_bytes(int nx, int ny) {
    const size_t N = (size_t)nx * ny, NE = (size_t)nx * (ny + 1) + (size_t)(nx + 1) * ny;
    size_t b = 0;
    b += 11 * align256(N * sizeof(double));      // H C S1H S1C S2H S2C LH LC T phi rate
    b += align256(18 * N * sizeof(double));      // rec
    b += align256(N);                            // flags
    b += 2 * align256(NE * kNQ * sizeof(double));// vsn udn
    b += align256(4 * NE * sizeof(double));      // face
    b += align256(sizeof(StageTables));
    return b;
}

cudaEvent_t prof_event(mp_batch* b) {
    if (b->ev_used == b->ev_pool.size()) { cudaEvent_t e; cudaEventCreate(&e); b->ev_pool.push_back(e); }
    return b->ev_pool[b->ev_used++];
}
template <class F>
void timed(mp_batch* b, int kind, F&& f) {
    if (!b->profile) { f(); return; }
    cudaEventRecord(prof_event(b), b->stream);
    f();
    cudaEventRecord(prof_event(b), b->stream);
    b->ev_kind.push_back(kind);
}
void harvest(mp_batch* b) {
    for (size_t k = 0; k < b->ev_kind.size(); ++k) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, b->ev_pool[2 * k], b->ev_pool[2 * k + 1]) == cudaSuccess) {
            b->kern_ms[b->ev_kind[k]] += ms;
            b->kern_n[b->ev_kind[k]] += 1;
        }
    }
    b->ev_kind.clear();
    b->ev_used = 0;
}

mp_status alloc_instance(mp_batch* b, MPInstance& in, const mp_mesh_desc& m) {
    in.mesh = m; in.nx = m.nx; in.ny = m.ny;
    in.N = (size_t)m.nx * m.ny;
    in.NE = (size_t)m.nx * (m.ny + 1) + (size_t)(m.nx + 1) * m.ny;
    const int tb = build_stage_tables(m.nx, m.ny, m.x0, m.x1, m.y0, m.y1, in.host_tab);
    if (tb) { set_error("stencil table construction failed"); return (mp_status)tb; }
    in.bytes = instance_bytes(m.nx, m.ny);
    MP_CUDA(cudaMallocAsync(&in.arena, in.bytes, b->stream));
    unsigned char* p = static_cast<unsigned char*>(in.arena);
    auto take = [&](size_t bytes) { void* r = p; p += align256(bytes); return r; };
    const size_t N = in.N, NE = in.NE;
    double** dbl[] = {&in.H, &in.C, &in.S1H, &in.S1C, &in.S2H, &in.S2C, &in.LH, &in.LC, &in.T, &in.phi, &in.rate};
    for (double** q : dbl) *q = static_cast<double*>(take(N * sizeof(double)));
    in.rec = static_cast<double*>(take(18 * N * sizeof(double)));
    in.flags = static_cast<unsigned char*>(take(N));
    in.vsn = static_cast<double*>(take(NE * kNQ * sizeof(double)));
    in.udn = static_cast<double*>(take(NE * kNQ * sizeof(double)));
    in.face = static_cast<double*>(take(4 * NE * sizeof(double)));
    in.tab = static_cast<StageTables*>(take(sizeof(StageTables)));
    MP_CUDA(cudaMemcpyAsync(in.tab, &in.host_tab, sizeof(StageTables), cudaMemcpyHostToDevice, b->stream));
    MP_CUDA(cudaMemsetAsync(in.vsn, 0, NE * kNQ * sizeof(double), b->stream));
    MP_CUDA(cudaMemsetAsync(in.udn, 0, NE * kNQ * sizeof(double), b->stream));
    MP_CUDA(cudaStreamSynchronize(b->stream));   // the copy source is the instance record, which a later add may move
    in.used = true;
    in.time = 0.0; in.accepted = 0; in.have_L = false; in.status = 0;
    b->bytes_in_use += in.bytes;
    b->dirty = true;
    return MP_OK;
}

// An instance on a general quad mesh: the arena of alloc_instance (its
// uniform-table slot unused) and the per-cell tables built on the GPU, as
// mp_transport_create_quads builds them.
mp_status alloc_quad_instance(mp_batch* b, MPInstance& in, const mp_mesh_desc& m, const double* xy) {
    long long bad = -1;
    if (validate_quads(m.nx, m.ny, xy, &bad)) {
        set_error("Mesh has non-real/non-finite coordinates or an inverted, degenerate, or nearly singular "
                  "quadrilateral (cell %lld)", bad);
        return MP_ERR_ARG_WRONG;
    }
    QuadTables qt;
    const int qs = build_quad_tables(m.nx, m.ny, xy, 0, qt, 0, m.ny, false);
    if (qs) { set_error("per-cell stencil table construction failed"); return (mp_status)qs; }
    in.mesh = m; in.nx = m.nx; in.ny = m.ny;
    in.N = (size_t)m.nx * m.ny;
    in.NE = (size_t)m.nx * (m.ny + 1) + (size_t)(m.nx + 1) * m.ny;
    in.bytes = instance_bytes(m.nx, m.ny);
    MP_CUDA(cudaMallocAsync(&in.arena, in.bytes, b->stream));
    unsigned char* p = static_cast<unsigned char*>(in.arena);
    auto take = [&](size_t bytes) { void* r = p; p += align256(bytes); return r; };
    const size_t N = in.N, NE = in.NE;
    double** dbl[] = {&in.H, &in.C, &in.S1H, &in.S1C, &in.S2H, &in.S2C, &in.LH, &in.LC, &in.T, &in.phi, &in.rate};
    for (double** q : dbl) *q = static_cast<double*>(take(N * sizeof(double)));
    in.rec = static_cast<double*>(take(18 * N * sizeof(double)));
    in.flags = static_cast<unsigned char*>(take(N));
    in.vsn = static_cast<double*>(take(NE * kNQ * sizeof(double)));
    in.udn = static_cast<double*>(take(NE * kNQ * sizeof(double)));
    in.face = static_cast<double*>(take(4 * NE * sizeof(double)));
    in.tab = nullptr;
    MP_CUDA(cudaMemsetAsync(in.vsn, 0, NE * kNQ * sizeof(double), b->stream));
    MP_CUDA(cudaMemsetAsync(in.udn, 0, NE * kNQ * sizeof(double), b->stream));
    cudaError_t ce = cudaSuccess;
    const int gs = upload_quad_tables(m.nx, m.ny, xy, qt, 0, m.ny, b->stream, &in.qbuf, in.qdev, &ce);
    if (gs) {
        cudaFreeAsync(in.arena, b->stream);
        cudaStreamSynchronize(b->stream);
        if (in.qbuf) cudaFree(in.qbuf);
        in = MPInstance{};
        if (gs == MP_ERR_ARG_WRONG) {
            set_error("per-cell stencil table construction failed (singular stencil or degenerate cell)");
            return MP_ERR_ARG_WRONG;
        }
        return cuda_status(ce, "mp_batch_add_quads");
    }
    in.qbytes = ((size_t)(kQG0 + kQS9 + kQT4 + kQS4 + kQGeo) * N + qt.xy.size() + qt.spacing.size()) * sizeof(double);
    in.cell_area = in.qdev.geo + 3 * N;
    in.quad = true;
    in.used = true;
    in.time = 0.0; in.accepted = 0; in.have_L = false; in.status = 0;
    b->bytes_in_use += in.bytes + in.qbytes;
    if (!b->has_quads) { b->has_quads = true; b->gen += 1; }
    b->dirty = true;
    return MP_OK;
}

void free_instance(mp_batch* b, MPInstance& in) {
    if (in.arena) cudaFreeAsync(in.arena, b->stream);
    if (in.src_arena) cudaFreeAsync(in.src_arena, b->stream);
    if (in.qbuf) {
        cudaStreamSynchronize(b->stream);
        cudaFree(in.qbuf);
    }
    b->bytes_in_use -= in.bytes + in.src_bytes + in.qbytes;
    in = MPInstance{};
    b->dirty = true;
}

// Grow-only device array: at least `need` entries, with headroom; *grown is
// set when the array moved (the captured graph must then be captured again).
template <class T>
mp_status grow(T** p, int& cap, int need, cudaStream_t s, bool* grown) {
    if (*p && need <= cap) return MP_OK;
    if (*p) cudaFreeAsync(*p, s);
    *p = nullptr;
    const int n = std::max(need + need / 2, 64);
    MP_CUDA(cudaMallocAsync((void**)p, (size_t)n * sizeof(T), s));
    cap = n;
    *grown = true;
    return MP_OK;
}

// Rebuild per-instance argument records, work maps and partial offsets.
template <class R>
mp_status rebuild_args(mp_batch* b, int slots) {
    std::vector<InstArgs<R>> args[NKIND];
    for (int k = 0; k < NKIND; ++k) args[k].resize(slots);
    std::vector<QuadStageArgs> qargs[NKIND];
    for (int k = 0; k < NKIND; ++k) qargs[k].resize(slots);
    std::vector<Work> wqr, wqp, wqf;
    std::vector<AxpyArgs> ax(slots);
    std::vector<CommitArgs> cm(slots);
    std::vector<int> part_off(slots, 0), part_cnt(slots, 0);
    std::vector<Work> wr, wp, wf, ws;
    int parts = 0;
    const Tuning tu = b->tune;
    for (int i = 0; i < slots; ++i) {
        MPInstance& in = b->inst[i];
        if (!in.used) continue;
        Tab<R> tb;
        tb.t = in.tab;
        const double area = in.quad ? 1.0 : in.host_tab.area;   // a quad mesh: per-cell areas
        const int nsum = (int)((in.N + kSumCells - 1) / kSumCells);
        part_off[i] = parts; part_cnt[i] = nsum;
        Partial* pp = nullptr;  // fixed below once the partial array exists
        (void)pp;
        for (int k = 0; k < NKIND; ++k) {
            const double* inH = k == KIND_P ? in.H : (k == KIND_B ? in.S1H : in.S2H);
            const double* inC = k == KIND_P ? in.C : (k == KIND_B ? in.S1C : in.S2C);
            double* outH = k == KIND_P ? in.LH : (k == KIND_B ? in.S2H : in.S1H);
            double* outC = k == KIND_P ? in.LC : (k == KIND_B ? in.S2C : in.S1C);
            InstArgs<R>& a = args[k][i];
            a.recon = ReconArgs<R>{in.nx, in.ny, tb, inH, inC, in.rec, in.flags, b->d_status + i, nullptr};
            a.phase = CellPhaseArgs<R>{in.nx, in.ny, tb, inH, inC, in.rec, in.flags, in.T, in.phi, b->d_status + i,
                                       0, 0, in.cvs_y, in.cud_y, in.srcH, in.srcR, in.srcS};
            a.face = FaceArgs<R>{in.nx, in.ny, tb, inH, inC, in.rec, in.flags, in.vsn, in.udn, in.face, b->d_status + i};
            const bool rk3 = b->opts.integrator == MP_SSPRK3;
            const double a0 = k == KIND_B ? (rk3 ? 0.75 : 0.5) : (1.0 / 3.0);
            const double a1 = k == KIND_B ? (rk3 ? 0.25 : 0.5) : (2.0 / 3.0);
            a.sum = SumArgs{in.nx, in.ny, area, 1.0 / area, in.face, inH, inC, in.H, in.C, outH, outC, in.rate,
                            k == KIND_P ? (int)SUM_STORE_L : (int)SUM_RK, a0, a1, 0.0, b->d_partial + parts,
                            b->d_dt + i, 0, 0, 0, -1, in.srcH, in.srcR, in.srcS, in.cell_area, nullptr, b->d_status + i};
            if (in.quad) {
                QuadStageArgs& q = qargs[k][i];
                q.nx = in.nx; q.ny = in.ny; q.gj0 = 0; q.gny = in.ny;
                q.H = inH; q.C = inC; q.rec = in.rec; q.flags = in.flags; q.T = in.T; q.phi = in.phi;
                q.vsn = in.vsn; q.udn = in.udn; q.face = in.face; q.status = b->d_status + i; q.theta = nullptr;
                q.q = in.qdev;
                q.src = SourcePtrs{in.cvs_y, in.cud_y, in.srcH, in.srcR, in.srcS};
            }
        }
        ax[i] = AxpyArgs{(int)in.N, in.H, in.C, in.LH, in.LC, in.S1H, in.S1C, b->d_dt + i, area,
                         b->d_partial + parts, in.cell_area};
        const bool rk3 = b->opts.integrator == MP_SSPRK3;
        cm[i] = CommitArgs{(int)in.N, rk3 ? in.S1H : in.S2H, rk3 ? in.S1C : in.S2C, in.H, in.C};
        if (in.quad) {
            // The quad kernels' tiles: 32x4 cells, 128 cells, 128 edges.
            for (int ty = 0; ty < in.ny; ty += 4)
                for (int tx = 0; tx < in.nx; tx += 32) wqr.push_back(Work{i, tx, ty, 0});
            for (size_t c = 0; c < in.N; c += 128) wqp.push_back(Work{i, (int)c, 0, 0});
            for (size_t e = 0; e < in.NE; e += 128) wqf.push_back(Work{i, (int)e, (int)std::min(in.NE, e + 128), 0});
        } else {
            for (int ty = 0; ty < in.ny; ty += tu.by)
                for (int tx = 0; tx < in.nx; tx += tu.bx * tu.cpt) wr.push_back(Work{i, tx, ty, 0});
            for (size_t c = 0; c < in.N; c += 128) wp.push_back(Work{i, (int)c, 0, 0});
            for (size_t e = 0; e < in.NE; e += 128) wf.push_back(Work{i, (int)e, (int)std::min(in.NE, e + 128), 0});
        }
        for (int s = 0; s < nsum; ++s) ws.push_back(Work{i, s * kSumCells, 0, s});
        parts += nsum;
    }
    (void)parts;
    cudaStream_t s = b->stream;
    // Per-slot records live in arrays of b->slots entries (allocated in rebuild).
    const int cap = b->slots;
    for (int k = 0; k < NKIND; ++k) args[k].resize(cap);
    for (int k = 0; k < NKIND; ++k) qargs[k].resize(cap);
    ax.resize(cap);
    cm.resize(cap);
    part_off.resize(cap, 0);
    part_cnt.resize(cap, 0);
    for (int k = 0; k < NKIND; ++k)
        MP_CUDA(cudaMemcpyAsync(b->d_args[k], args[k].data(), cap * sizeof(InstArgs<R>), cudaMemcpyHostToDevice, s));
    for (int k = 0; k < NKIND; ++k)
        MP_CUDA(cudaMemcpyAsync(b->d_qargs[k], qargs[k].data(), cap * sizeof(QuadStageArgs), cudaMemcpyHostToDevice, s));
    MP_CUDA(cudaMemcpyAsync(b->d_axpy, ax.data(), cap * sizeof(AxpyArgs), cudaMemcpyHostToDevice, s));
    MP_CUDA(cudaMemcpyAsync(b->d_commit, cm.data(), cap * sizeof(CommitArgs), cudaMemcpyHostToDevice, s));
    MP_CUDA(cudaMemcpyAsync(b->d_part_off, part_off.data(), cap * sizeof(int), cudaMemcpyHostToDevice, s));
    MP_CUDA(cudaMemcpyAsync(b->d_part_cnt, part_cnt.data(), cap * sizeof(int), cudaMemcpyHostToDevice, s));
    // Work lists, padded to their capacity with the sentinel slot.
    bool grown = false;
    b->n_wrecon = (int)wr.size(); b->n_wphase = (int)wp.size(); b->n_wface = (int)wf.size(); b->n_wsum = (int)ws.size();
    MP_TRY(grow(&b->d_wrecon, b->cap_wrecon, b->n_wrecon, s, &grown));
    MP_TRY(grow(&b->d_wphase, b->cap_wphase, b->n_wphase, s, &grown));
    MP_TRY(grow(&b->d_wface, b->cap_wface, b->n_wface, s, &grown));
    MP_TRY(grow(&b->d_wsum, b->cap_wsum, b->n_wsum, s, &grown));
    const Work pad{cap, 0, 0, 0};
    wr.resize(b->cap_wrecon, pad); wp.resize(b->cap_wphase, pad); wf.resize(b->cap_wface, pad); ws.resize(b->cap_wsum, pad);
    MP_CUDA(cudaMemcpyAsync(b->d_wrecon, wr.data(), wr.size() * sizeof(Work), cudaMemcpyHostToDevice, s));
    MP_CUDA(cudaMemcpyAsync(b->d_wphase, wp.data(), wp.size() * sizeof(Work), cudaMemcpyHostToDevice, s));
    MP_CUDA(cudaMemcpyAsync(b->d_wface, wf.data(), wf.size() * sizeof(Work), cudaMemcpyHostToDevice, s));
    MP_CUDA(cudaMemcpyAsync(b->d_wsum, ws.data(), ws.size() * sizeof(Work), cudaMemcpyHostToDevice, s));
    if (b->has_quads) {
        b->n_wqrec = (int)wqr.size(); b->n_wqphase = (int)wqp.size(); b->n_wqface = (int)wqf.size();
        MP_TRY(grow(&b->d_wqrec, b->cap_wqrec, b->n_wqrec, s, &grown));
        MP_TRY(grow(&b->d_wqphase, b->cap_wqphase, b->n_wqphase, s, &grown));
        MP_TRY(grow(&b->d_wqface, b->cap_wqface, b->n_wqface, s, &grown));
        wqr.resize(b->cap_wqrec, pad); wqp.resize(b->cap_wqphase, pad); wqf.resize(b->cap_wqface, pad);
        MP_CUDA(cudaMemcpyAsync(b->d_wqrec, wqr.data(), wqr.size() * sizeof(Work), cudaMemcpyHostToDevice, s));
        MP_CUDA(cudaMemcpyAsync(b->d_wqphase, wqp.data(), wqp.size() * sizeof(Work), cudaMemcpyHostToDevice, s));
        MP_CUDA(cudaMemcpyAsync(b->d_wqface, wqf.data(), wqf.size() * sizeof(Work), cudaMemcpyHostToDevice, s));
    }
    if (grown) b->gen += 1;
    MP_CUDA(cudaStreamSynchronize(s));   // host vectors go out of scope
    return MP_OK;
}

mp_status rebuild(mp_batch* b) {
    if (!b->dirty) return MP_OK;
    cudaStream_t s = b->stream;
    const int slots = (int)b->inst.size();
    // Per-slot arrays, with headroom; d_active has one more entry, the
    // sentinel slot named by padded work items, which stays 0.
    if (slots > b->slots || b->slots == 0) {
        for (void* p : {(void*)b->d_active, (void*)b->d_part_off, (void*)b->d_part_cnt, (void*)b->d_tot,
                        (void*)b->d_status, (void*)b->d_dt, (void*)b->d_axpy, (void*)b->d_commit, b->d_args[0],
                        b->d_args[1], b->d_args[2], b->d_qargs[0], b->d_qargs[1], b->d_qargs[2]})
            if (p) cudaFreeAsync(p, s);
        if (b->h_tot) cudaFreeHost(b->h_tot);
        if (b->h_status) cudaFreeHost(b->h_status);
        if (b->h_dt) cudaFreeHost(b->h_dt);
        if (b->h_active) cudaFreeHost(b->h_active);
        const int cap = std::max(slots + slots / 2, 8);
        MP_CUDA(cudaMallocAsync((void**)&b->d_active, (cap + 1) * sizeof(int), s));
        MP_CUDA(cudaMemsetAsync(b->d_active, 0, (cap + 1) * sizeof(int), s));
        MP_CUDA(cudaMallocAsync((void**)&b->d_part_off, cap * sizeof(int), s));
        MP_CUDA(cudaMallocAsync((void**)&b->d_part_cnt, cap * sizeof(int), s));
        MP_CUDA(cudaMallocAsync((void**)&b->d_tot, cap * sizeof(Totals), s));
        MP_CUDA(cudaMallocAsync((void**)&b->d_status, cap * sizeof(unsigned long long), s));
        MP_CUDA(cudaMemsetAsync(b->d_status, 0xff, cap * sizeof(unsigned long long), s));
        MP_CUDA(cudaMallocAsync((void**)&b->d_dt, cap * sizeof(double), s));
        MP_CUDA(cudaMallocAsync((void**)&b->d_axpy, cap * sizeof(AxpyArgs), s));
        MP_CUDA(cudaMallocAsync((void**)&b->d_commit, cap * sizeof(CommitArgs), s));
        for (int k = 0; k < NKIND; ++k) MP_CUDA(cudaMallocAsync(&b->d_args[k], cap * sizeof(InstArgs<double>), s));
        for (int k = 0; k < NKIND; ++k) MP_CUDA(cudaMallocAsync(&b->d_qargs[k], cap * sizeof(QuadStageArgs), s));
        MP_CUDA(cudaMallocHost((void**)&b->h_tot, cap * sizeof(Totals)));
        MP_CUDA(cudaMallocHost((void**)&b->h_status, cap * sizeof(unsigned long long)));
        MP_CUDA(cudaMallocHost((void**)&b->h_dt, cap * sizeof(double)));
        MP_CUDA(cudaMallocHost((void**)&b->h_active, cap * sizeof(int)));
        for (int i = 0; i < cap; ++i) b->h_active[i] = 0;
        b->slots = cap;
        b->gen += 1;
    }
    int parts = 0;
    for (const MPInstance& in : b->inst) if (in.used) parts += (int)((in.N + kSumCells - 1) / kSumCells);
    if (parts > b->partial_cap) {
        if (b->d_partial) cudaFreeAsync(b->d_partial, s);
        const int n = std::max(parts + parts / 2, 64);
        MP_CUDA(cudaMallocAsync((void**)&b->d_partial, n * sizeof(Partial), s));
        b->partial_cap = n;
        b->gen += 1;
    }
    MP_TRY(rebuild_args<double>(b, slots));
    b->dirty = false;
    return MP_OK;
}

mp_status set_active(mp_batch* b, const std::vector<int>& act) {
    const int slots = (int)b->inst.size();
    for (int i = 0; i < slots; ++i) b->h_active[i] = act[i];
    MP_CUDA(cudaMemcpyAsync(b->d_active, b->h_active, slots * sizeof(int), cudaMemcpyHostToDevice, b->stream));
    return MP_OK;
}

template <class R>
void launch_kind(mp_batch* b, int kind) {
    cudaStream_t s = b->stream;
    const InstArgs<R>* args = static_cast<const InstArgs<R>*>(b->d_args[kind]);
    const Tuning tu = b->tune;
    // Grids cover the work lists' capacities (padded items exit at once).
    timed(b, 0, [&] { batch_recon_kernel<R><<<b->cap_wrecon, dim3(tu.bx, tu.by), 0, s>>>(args, b->d_wrecon, b->d_active, b->ph, tu.cpt); });
    if (b->ph.source) timed(b, 1, [&] { batch_phase_kernel<R, true><<<b->cap_wphase, 128, 0, s>>>(args, b->d_wphase, b->d_active, b->ph); });
    else timed(b, 1, [&] { batch_phase_kernel<R, false><<<b->cap_wphase, 128, 0, s>>>(args, b->d_wphase, b->d_active, b->ph); });
    timed(b, 2, [&] { batch_face_kernel<R><<<b->cap_wface, 128, 0, s>>>(args, b->d_wface, b->d_active, b->ph); });
    if (b->ph.diffusion)
        timed(b, 2, [&] { batch_diffusion_kernel<R><<<b->cap_wface, 128, 0, s>>>(args, b->d_wface, b->d_active, b->ph); });
    if (b->has_quads) {
        // General quad meshes: reconstruction, limiter, cell phase (the wet
        // flags the faces read), faces; the sums below cover every instance.
        const QuadStageArgs* qa = static_cast<const QuadStageArgs*>(b->d_qargs[kind]);
        timed(b, 0, [&] { batch_quad_weno_kernel<<<b->cap_wqrec, dim3(32, 4), 0, s>>>(qa, b->d_wqrec, b->d_active); });
        timed(b, 0, [&] { batch_quad_limit_kernel<<<b->cap_wqrec, dim3(32, 4), 0, s>>>(qa, b->d_wqrec, b->d_active, b->ph); });
        timed(b, 1, [&] { batch_quad_phase_kernel<<<b->cap_wqphase, 128, 0, s>>>(qa, b->d_wqphase, b->d_active, b->ph); });
        timed(b, 2, [&] { batch_quad_face_kernel<<<b->cap_wqface, 128, 0, s>>>(qa, b->d_wqface, b->d_active, b->ph); });
        if (b->ph.diffusion)
            timed(b, 2, [&] { batch_quad_diffusion_kernel<<<b->cap_wqface, 128, 0, s>>>(qa, b->d_wqface, b->d_active, b->ph); });
        count_launch(b->ph.diffusion ? 5 : 4);
    }
    if (b->ph.source) timed(b, 3, [&] { batch_sum_kernel<R, true><<<b->cap_wsum, kRedBlock, 0, s>>>(args, b->d_wsum, b->d_active); });
    else timed(b, 3, [&] { batch_sum_kernel<R, false><<<b->cap_wsum, kRedBlock, 0, s>>>(args, b->d_wsum, b->d_active); });
    timed(b, 4, [&] { batch_reduce_kernel<<<b->slots, 1024, 0, s>>>(b->d_partial, b->d_part_off, b->d_part_cnt, b->d_active, b->d_tot); });
    count_launch(5);
}

// Stage of one kind on the active instances; totals and status to the host.
mp_status run_stage(mp_batch* b, int kind, const std::vector<int>& act) {
    NvtxRange range("mp_batch stage");
    MP_TRY(set_active(b, act));
    const int slots = (int)b->inst.size();
    MP_CUDA(cudaMemsetAsync(b->d_status, 0xff, slots * sizeof(unsigned long long), b->stream));
    launch_kind<double>(b, kind);
    MP_CUDA(cudaGetLastError());
    MP_CUDA(cudaMemcpyAsync(b->h_tot, b->d_tot, slots * sizeof(Totals), cudaMemcpyDeviceToHost, b->stream));
    MP_CUDA(cudaMemcpyAsync(b->h_status, b->d_status, slots * sizeof(unsigned long long), cudaMemcpyDeviceToHost, b->stream));
    MP_CUDA(cudaStreamSynchronize(b->stream));
    b->host_syncs += 1;
    harvest(b);
    return MP_OK;
}

mp_status run_axpy(mp_batch* b, const std::vector<int>& act) {
    MP_TRY(set_active(b, act));
    const int slots = (int)b->inst.size();
    cudaStream_t s = b->stream;
    MP_CUDA(cudaMemcpyAsync(b->d_dt, b->h_dt, slots * sizeof(double), cudaMemcpyHostToDevice, s));
    timed(b, 4, [&] { batch_axpy_kernel<<<b->cap_wsum, kRedBlock, 0, s>>>(b->d_axpy, b->d_wsum, b->d_active); });
    timed(b, 4, [&] { batch_reduce_kernel<<<b->slots, 1024, 0, s>>>(b->d_partial, b->d_part_off, b->d_part_cnt, b->d_active, b->d_tot); });
    count_launch(2);
    MP_CUDA(cudaGetLastError());
    MP_CUDA(cudaMemcpyAsync(b->h_tot, b->d_tot, slots * sizeof(Totals), cudaMemcpyDeviceToHost, s));
    MP_CUDA(cudaStreamSynchronize(s));
    b->host_syncs += 1;
    harvest(b);
    return MP_OK;
}

int status_code(unsigned long long v) { return v == ~0ULL ? 0 : (int)(v & 0xff); }

bool admissible_tot(const Totals& t, double Xe) {
    return t.nonfinite == 0.0 && t.Hmin >= 0.0 && t.Cmin >= 0.0 && t.Cmax <= Xe;
}

// With the adiabatic source on, every instance needs its cell-point
// velocities (the single-instance path's rule).
mp_status check_sources(const mp_batch* b) {
    if (!b->ph.source) return MP_OK;
    for (size_t i = 0; i < b->inst.size(); ++i)
        if (b->inst[i].used && !b->inst[i].cvs_y) {
            set_error("instance %zu: the adiabatic source (alpha0 != 0) needs the flow velocities at the cell "
                      "quadrature points (mp_batch_set_cell_velocity)", i);
            return MP_ERR_ARG_WRONGSTATE;
        }
    return MP_OK;
}

// L(U^n) for instances that lack it.
mp_status eval_missing(mp_batch* b) {
    const int slots = (int)b->inst.size();
    std::vector<int> act(slots, 0);
    bool any = false;
    for (int i = 0; i < slots; ++i) {
        const MPInstance& in = b->inst[i];
        if (in.used && !in.status && !in.have_L) { act[i] = 1; any = true; }
    }
    if (!any) return MP_OK;
    MP_TRY(run_stage(b, KIND_P, act));
    for (int i = 0; i < slots; ++i) {
        if (!act[i]) continue;
        MPInstance& in = b->inst[i];
        const int st = status_code(b->h_status[i]);
        if (st) { in.status = st; continue; }
        if (!std::isfinite(b->h_tot[i].maxRate)) { in.status = MP_ERR_FP; continue; }
        in.cur = b->h_tot[i];
        in.have_L = true;
    }
    return MP_OK;
}

// One accepted step of every healthy instance (the reference's loop per instance).
mp_status step_all(mp_batch* b, std::vector<mp_step_report>& reps) {
    NvtxRange range("mp_batch step (host loop)");
    MP_TRY(check_sources(b));
    MP_TRY(rebuild(b));
    MP_TRY(eval_missing(b));
    const int slots = (int)b->inst.size();
    const mp_transport_opts& o = b->opts;
    const double Xe = o.material.Xe;
    const bool rk3 = o.integrator == MP_SSPRK3;
    reps.assign(slots, mp_step_report{});
    std::vector<double> dt(slots, 0.0), start(slots, 0.0), courant(slots, 0.0);
    std::vector<int> retries(slots, 0), pending(slots, 0), done(slots, 0);
    std::vector<Totals> first(slots), second(slots), third(slots);
    std::vector<double> remaining(slots, INFINITY);
    for (int i = 0; i < slots; ++i) {
        MPInstance& in = b->inst[i];
        if (!in.used || in.status) continue;
        if (finished(in)) { in.time = in.t_end; continue; }
        first[i] = in.cur;
        remaining[i] = in.t_end - in.time;
        const double cap = in.accepted == 0 ? o.dt_initial : o.dt_max;
        const double limit = in.cur.maxRate > 0 ? o.cfl / in.cur.maxRate : o.dt_max;
        dt[i] = std::min(std::min(remaining[i], cap), limit);
        start[i] = in.time;
        pending[i] = 1;
    }
    for (;;) {
        bool any = false;
        for (int i = 0; i < slots; ++i) {
            if (!pending[i]) continue;
            if (!(dt[i] >= std::min(remaining[i], o.dt_min) && retries[i] < 40)) { b->inst[i].status = MP_ERR_NOT_CONVERGED; pending[i] = 0; continue; }
            b->h_dt[i] = dt[i];
            any = true;
        }
        if (!any) break;
        MP_TRY(run_axpy(b, pending));
        std::vector<int> valid(slots, 0);
        for (int i = 0; i < slots; ++i) if (pending[i]) valid[i] = admissible_tot(b->h_tot[i], Xe);
        MP_TRY(run_stage(b, KIND_B, valid));
        for (int i = 0; i < slots; ++i) {
            if (!valid[i]) continue;
            const int st = status_code(b->h_status[i]);
            if (st || !std::isfinite(b->h_tot[i].maxRate)) { b->inst[i].status = st ? st : MP_ERR_FP; valid[i] = 0; pending[i] = 0; continue; }
            second[i] = b->h_tot[i];
            courant[i] = dt[i] * std::max(first[i].maxRate, second[i].maxRate);
            valid[i] = courant[i] <= o.cfl * (1 + 1e-12) && admissible_tot(second[i], Xe);
        }
        if (rk3) {
            MP_TRY(run_stage(b, KIND_C, valid));
            for (int i = 0; i < slots; ++i) {
                if (!valid[i]) continue;
                const int st = status_code(b->h_status[i]);
                if (st || !std::isfinite(b->h_tot[i].maxRate)) { b->inst[i].status = st ? st : MP_ERR_FP; valid[i] = 0; pending[i] = 0; continue; }
                third[i] = b->h_tot[i];
                courant[i] = dt[i] * std::max(std::max(first[i].maxRate, second[i].maxRate), third[i].maxRate);
                valid[i] = courant[i] <= o.cfl * (1 + 1e-12) && admissible_tot(third[i], Xe);
            }
        }
        for (int i = 0; i < slots; ++i) {
            if (!pending[i]) continue;
            if (valid[i]) { done[i] = 1; pending[i] = 0; }
            else { dt[i] *= 0.5; ++retries[i]; }
        }
    }
    // Balance check and commit (evolve.cpp:486-499).
    cudaStream_t s = b->stream;
    for (int i = 0; i < slots; ++i) {
        if (!done[i]) continue;
        MPInstance& in = b->inst[i];
        const Totals fin = rk3 ? third[i] : second[i];
        const Totals& f = first[i];
        const Totals& sd = second[i];
        double repH, repC, repS, bH, bC;
        if (rk3) {
            repH = (f.bH + sd.bH) / 6 + third[i].bH * (2.0 / 3.0);
            repC = (f.bC + sd.bC) / 6 + third[i].bC * (2.0 / 3.0);
            repS = (f.sH + sd.sH) / 6 + third[i].sH * (2.0 / 3.0);
            bH = fin.HI - f.HI + dt[i] * (repH - repS);
            bC = fin.CI - f.CI + dt[i] * repC;
        } else {
            repH = .5 * (f.bH + sd.bH);
            repC = .5 * (f.bC + sd.bC);
            repS = .5 * (f.sH + sd.sH);
            bH = fin.HI - f.HI + .5 * dt[i] * (f.bH + sd.bH - f.sH - sd.sH);
            bC = fin.CI - f.CI + .5 * dt[i] * (f.bC + sd.bC);
        }
        if (!(std::fabs(bH) < 1e-10 * std::max(1.0, std::fabs(first[i].HI)) && std::fabs(bC) < 1e-10)) {
            in.status = MP_ERR_PLIB;
            done[i] = 0;
            continue;
        }
        double* nH = rk3 ? in.S1H : in.S2H;
        double* nC = rk3 ? in.S1C : in.S2C;
        MP_CUDA(cudaMemcpyAsync(in.H, nH, in.N * sizeof(double), cudaMemcpyDeviceToDevice, s));
        MP_CUDA(cudaMemcpyAsync(in.C, nC, in.N * sizeof(double), cudaMemcpyDeviceToDevice, s));
        in.time = start[i] + dt[i];
        if (std::isfinite(in.t_end) && in.t_end - in.time <= 32 * 2.220446049250313e-16 * std::max(1.0, std::fabs(in.t_end)))
            in.time = in.t_end;
        in.have_L = false;
        mp_step_report& r = reps[i];
        r.retries = retries[i]; r.dt = dt[i]; r.time = in.time; r.courant = courant[i];
        r.boundaryH = repH; r.boundaryC = repC; r.sourceH = repS; r.balanceH = bH; r.balanceC = bC;
        r.H_integral = fin.HI; r.C_integral = fin.CI;
    }
    MP_TRY(eval_missing(b));
    for (int i = 0; i < slots; ++i) {
        MPInstance& in = b->inst[i];
        if (!in.used) continue;
        if (done[i] && !in.status) {
            ++in.accepted;
            reps[i].maxRate = in.cur.maxRate;
            reps[i].divergence = in.cur.divergence;
        }
        reps[i].status = in.status;
    }
    return MP_OK;
}

// Autotuner: time one P-stage over the whole batch for each candidate tile
// shape / cells-per-thread of the reconstruction kernel; keep the fastest.
mp_status autotune(mp_batch* b, int reps, double* best_ms) {
    const Tuning cands[] = {{32, 4, 1}, {32, 2, 1}, {64, 2, 1}, {16, 8, 1}, {128, 1, 1}, {32, 4, 2}, {32, 2, 2}, {64, 1, 2}};
    const int slots = (int)b->inst.size();
    std::vector<int> act(slots, 0);
    for (int i = 0; i < slots; ++i) act[i] = b->inst[i].used && !b->inst[i].status;
    double best = 1e300;
    Tuning pick = b->tune;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0); cudaEventCreate(&e1);
    for (const Tuning& c : cands) {
        b->tune = c;
        b->dirty = true;
        MP_TRY(rebuild(b));
        MP_TRY(set_active(b, act));
        launch_kind<double>(b, KIND_P);   // warm-up
        cudaEventRecord(e0, b->stream);
        for (int r = 0; r < reps; ++r) launch_kind<double>(b, KIND_P);
        cudaEventRecord(e1, b->stream);
        MP_CUDA(cudaEventSynchronize(e1));
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best) { best = ms; pick = c; }
    }
    cudaEventDestroy(e0); cudaEventDestroy(e1);
    b->tune = pick;
    b->dirty = true;
    MP_TRY(rebuild(b));
    b->gen += 1;      // the captured graph has the block shape of the old tile
    // the timing runs overwrote L and T/phi of every instance: recompute L(U^n)
    for (MPInstance& in : b->inst) in.have_L = false;
    if (best_ms) *best_ms = best / reps;
    return MP_OK;
}

// ------------------------------------------------------- device-resident steps

constexpr int kGraphChunk = 64;        // steps per graph launch (report rows)

StepOpts step_opts(const mp_batch* b) {
    const mp_transport_opts& o = b->opts;
    StepOpts so{};
    so.cfl = o.cfl; so.dt_initial = o.dt_initial; so.dt_max = o.dt_max; so.dt_min = o.dt_min; so.Xe = o.material.Xe;
    so.rk3 = o.integrator == MP_SSPRK3;
    so.fixed = 0;
    so.snap_end = 1; so.end_reports = 0; so.restore_time = 0;
    return so;
}

// Current leaf nodes of a capture (the dependencies of the next node).
mp_status capture_leaves(cudaStream_t s, std::vector<cudaGraphNode_t>& out) {
    cudaStreamCaptureStatus cs;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    MP_CUDA(cudaStreamGetCaptureInfo(s, &cs, nullptr, nullptr, &deps, &nd));
    out.assign(deps, deps + nd);
    return MP_OK;
}

// A conditional WHILE node in `g` after `deps`; its body graph in *body.
mp_status add_while(cudaGraph_t g, const std::vector<cudaGraphNode_t>& deps, cudaGraphConditionalHandle h,
                    cudaGraphNode_t* node, cudaGraph_t* body) {
    cudaGraphNodeParams p{};
    p.type = cudaGraphNodeTypeConditional;
    p.conditional.handle = h;
    p.conditional.type = cudaGraphCondTypeWhile;
    p.conditional.size = 1;
    MP_CUDA(cudaGraphAddNode(node, g, deps.empty() ? nullptr : deps.data(), deps.size(), &p));
    *body = p.conditional.phGraph_out[0];
    return MP_OK;
}

// The graph of up to kGraphChunk steps of every instance:
//   WHILE run:  begin -> WHILE attempt: {attempt, axpy, reduce, gate,
//               stage B, control [, stage C, control]} -> commit, copy,
//               stage P (L(U^{n+1})), control (run condition).
template <class R>
mp_status capture_graph(mp_batch* b, cudaGraph_t* out) {
    cudaStream_t s = b->stream;
    const int slots = b->slots;          // control records of every slot of the capacity
    const StepOpts so = step_opts(b);
    const bool rk3 = so.rk3 != 0;
    cudaGraph_t g = nullptr;
    MP_CUDA(cudaGraphCreate(&g, 0));
    *out = g;
    cudaGraphConditionalHandle run, attempt;
    MP_CUDA(cudaGraphConditionalHandleCreate(&run, g, 1, cudaGraphCondAssignDefault));
    cudaGraphNode_t run_node, attempt_node;
    cudaGraph_t step_body, attempt_body;
    MP_TRY(add_while(g, {}, run, &run_node, &step_body));
    MP_CUDA(cudaGraphConditionalHandleCreate(&attempt, step_body, 0, 0));
    const cudaStreamCaptureMode mode = cudaStreamCaptureModeThreadLocal;
    cudaGraph_t tmp;
    // Step begin.
    MP_CUDA(cudaStreamBeginCaptureToGraph(s, step_body, nullptr, nullptr, 0, mode));
    ctl_begin_kernel<<<1, kCtlThreads, 0, s>>>(b->d_ctl, slots, so, b->d_hdr, b->d_rep, attempt);
    std::vector<cudaGraphNode_t> leaves;
    MP_TRY(capture_leaves(s, leaves));
    MP_CUDA(cudaStreamEndCapture(s, &tmp));
    MP_TRY(add_while(step_body, leaves, attempt, &attempt_node, &attempt_body));
    // One attempt.
    MP_CUDA(cudaStreamBeginCaptureToGraph(s, attempt_body, nullptr, nullptr, 0, mode));
    ctl_attempt_kernel<<<1, kCtlThreads, 0, s>>>(b->d_ctl, slots, so, b->d_hdr, b->d_active, b->d_dt);
    batch_axpy_kernel<<<b->cap_wsum, kRedBlock, 0, s>>>(b->d_axpy, b->d_wsum, b->d_active);
    batch_reduce_kernel<<<b->slots, 1024, 0, s>>>(b->d_partial, b->d_part_off, b->d_part_cnt, b->d_active, b->d_tot);
    ctl_after_axpy_kernel<<<1, kCtlThreads, 0, s>>>(b->d_ctl, slots, so, b->d_tot, b->d_status, b->d_active);
    launch_kind<R>(b, KIND_B);
    ctl_after_stage_kernel<<<1, kCtlThreads, 0, s>>>(b->d_ctl, slots, so, b->d_tot, b->d_status, b->d_active, 2,
                                                      rk3 ? 0 : 1, b->d_hdr, attempt);
    if (rk3) {
        launch_kind<R>(b, KIND_C);
        ctl_after_stage_kernel<<<1, kCtlThreads, 0, s>>>(b->d_ctl, slots, so, b->d_tot, b->d_status, b->d_active, 3, 1,
                                                          b->d_hdr, attempt);
    }
    MP_CUDA(cudaStreamEndCapture(s, &tmp));
    // Commit and L(U^{n+1}).
    MP_CUDA(cudaStreamBeginCaptureToGraph(s, step_body, &attempt_node, nullptr, 1, mode));
    ctl_commit_kernel<<<1, kCtlThreads, 0, s>>>(b->d_ctl, slots, so, b->d_hdr, b->d_rep, b->d_status, b->d_active);
    batch_commit_kernel<<<b->cap_wsum, kRedBlock, 0, s>>>(b->d_commit, b->d_wsum, b->d_active);
    launch_kind<R>(b, KIND_P);
    ctl_after_rhs_kernel<<<1, kCtlThreads, 0, s>>>(b->d_ctl, slots, so, b->d_tot, b->d_status, b->d_rep, b->d_hdr, 0,
                                                    run);
    MP_CUDA(cudaStreamEndCapture(s, &tmp));
    MP_CUDA(cudaGetLastError());
    return MP_OK;
}

void release_graph(mp_batch* b) {
    if (b->graph_exec) cudaGraphExecDestroy(b->graph_exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->graph_exec = nullptr;
    b->graph = nullptr;
    b->graph_gen = 0;
}

mp_status ensure_graph(mp_batch* b) {
    cudaStream_t s = b->stream;
    if (b->slots != b->graph_slots) {
        for (void* p : {(void*)b->d_ctl, (void*)b->d_hdr, (void*)b->d_rep}) if (p) cudaFreeAsync(p, s);
        for (void* p : {(void*)b->h_ctl, (void*)b->h_hdr, (void*)b->h_rep}) if (p) cudaFreeHost(p);
        const int cap = b->slots;
        MP_CUDA(cudaMallocAsync((void**)&b->d_ctl, cap * sizeof(InstCtl), s));
        MP_CUDA(cudaMallocAsync((void**)&b->d_hdr, sizeof(CtlHeader), s));
        MP_CUDA(cudaMallocAsync((void**)&b->d_rep, (size_t)kGraphChunk * cap * sizeof(mp_step_report), s));
        MP_CUDA(cudaMallocHost((void**)&b->h_ctl, cap * sizeof(InstCtl)));
        MP_CUDA(cudaMallocHost((void**)&b->h_hdr, sizeof(CtlHeader)));
        MP_CUDA(cudaMallocHost((void**)&b->h_rep, (size_t)kGraphChunk * cap * sizeof(mp_step_report)));
        b->graph_slots = cap;
        b->gen += 1;
    }
    if (b->graph_exec && b->graph_gen == b->gen) return MP_OK;
    release_graph(b);
    b->stage_kernels = 5 + (b->ph.diffusion ? 1 : 0) + (b->has_quads ? (b->ph.diffusion ? 5 : 4) : 0);
    // Capture on a private stream (the caller's may be the legacy default
    // stream, which cannot be captured); the graph runs on the caller's.
    cudaStream_t cap = nullptr;
    MP_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    cudaStream_t user = b->stream;
    b->stream = cap;
    g_capturing = true;
    const mp_status st = capture_graph<double>(b, &b->graph);
    g_capturing = false;
    cudaStreamCaptureStatus cs;
    if (cudaStreamIsCapturing(cap, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone) {
        cudaGraph_t tmp;
        cudaStreamEndCapture(cap, &tmp);
    }
    b->stream = user;
    cudaStreamDestroy(cap);
    if (st != MP_OK) { release_graph(b); return st; }
    MP_CUDA(cudaGraphInstantiate(&b->graph_exec, b->graph, 0));
    b->graph_gen = b->gen;
    b->captures += 1;
    return MP_OK;
}

// nsteps steps of every instance on the device: one graph launch and one host
// wait per kGraphChunk steps. Same decisions and results as step_all.
mp_status graph_steps(mp_batch* b, int nsteps, mp_step_report* reports) {
    NvtxRange range("mp_batch steps (device-resident graph)");
    MP_TRY(check_sources(b));
    MP_TRY(rebuild(b));
    MP_TRY(eval_missing(b));
    MP_TRY(ensure_graph(b));
    const int slots = (int)b->inst.size();
    const int cap = b->slots;            // control records and report rows cover the capacity
    cudaStream_t s = b->stream;
    for (int done = 0; done < nsteps; done += kGraphChunk) {
        const int chunk = std::min(kGraphChunk, nsteps - done);
        for (int i = 0; i < cap; ++i) {
            InstCtl& c = b->h_ctl[i];
            c = InstCtl{};
            if (i >= slots) continue;
            const MPInstance& in = b->inst[i];
            c.used = in.used ? 1 : 0;
            c.time = in.time; c.t_end = in.t_end;
            c.accepted = in.accepted; c.status = in.status; c.have_L = in.have_L ? 1 : 0;
            c.cur = in.cur;
        }
        *b->h_hdr = CtlHeader{0, chunk, 0, 0, 0};
        MP_CUDA(cudaMemcpyAsync(b->d_ctl, b->h_ctl, cap * sizeof(InstCtl), cudaMemcpyHostToDevice, s));
        MP_CUDA(cudaMemcpyAsync(b->d_hdr, b->h_hdr, sizeof(CtlHeader), cudaMemcpyHostToDevice, s));
        MP_CUDA(cudaGraphLaunch(b->graph_exec, s));
        MP_CUDA(cudaMemcpyAsync(b->h_ctl, b->d_ctl, cap * sizeof(InstCtl), cudaMemcpyDeviceToHost, s));
        MP_CUDA(cudaMemcpyAsync(b->h_hdr, b->d_hdr, sizeof(CtlHeader), cudaMemcpyDeviceToHost, s));
        MP_CUDA(cudaMemcpyAsync(b->h_rep, b->d_rep, (size_t)chunk * cap * sizeof(mp_step_report),
                                cudaMemcpyDeviceToHost, s));
        MP_CUDA(cudaStreamSynchronize(s));
        b->host_syncs += 1;
        const CtlHeader h = *b->h_hdr;
        // Kernels the graph ran: per step 5 control/copy kernels and one
        // stage; per attempt 4 control/axpy kernels and one or two stages.
        const int per_attempt = 4 + (b->stage_kernels + 1) * (b->opts.integrator == MP_SSPRK3 ? 2 : 1);
        count_launch((unsigned long long)h.step * (3 + b->stage_kernels + 1) +
                     (unsigned long long)h.total_attempts * per_attempt);
        for (int i = 0; i < slots; ++i) {
            MPInstance& in = b->inst[i];
            if (!in.used) continue;
            const InstCtl& c = b->h_ctl[i];
            in.time = c.time; in.accepted = c.accepted; in.status = c.status; in.have_L = c.have_L != 0;
            in.cur = c.cur;
        }
        if (reports)
            for (int k = 0; k < chunk; ++k)
                std::memcpy(reports + (size_t)(done + k) * slots, b->h_rep + (size_t)k * cap,
                            (size_t)slots * sizeof(mp_step_report));
    }
    return MP_OK;
}

}  // namespace
}  // namespace mp

// -------------------------------------------------------------------- C ABI

extern "C" mp_status mp_batch_create(const mp_mesh_desc* meshes, int count, const mp_transport_opts* opts,
                                     mp_stream_t stream, mp_batch** out) {
    using namespace mp;
    if (!opts || !out || count < 0 || (count > 0 && !meshes)) { set_error("null argument"); return MP_ERR_ARG_WRONG; }
    mp_derived der;
    MP_TRY(validate_opts(*opts, &der));
    mp_batch* b = new mp_batch;
    b->opts = *opts; b->der = der;
    b->stream = (cudaStream_t)stream;
    b->ph.k = phase_const(opts->material, der);
    b->ph.sk = stage_const(b->ph.k);
    if (eutectic_temperature(b->ph.k, opts->pressure, b->ph.Tep)) { delete b; set_error("pressure must be finite"); return MP_ERR_ARG_OUTOFRANGE; }
    b->ph.theta = opts->theta; b->ph.inflowH = opts->inflow_H; b->ph.inflowC = opts->inflow_C;
    b->ph.Hpol = opts->H_policy; b->ph.Cpol = opts->C_policy; b->ph.lf_global = opts->lf_global;
    b->ph.lf_speed = opts->lf_global_speed;
    b->ph.kappa = opts->diffusivity;
    for (int w = 0; w < 4; ++w) { b->ph.wall_type[w] = 0; b->ph.wall_value[w] = 0.0; }
    b->ph.diffusion = opts->diffusivity > 0.0;
    b->ph.litho = 0; b->ph.tep_a = b->ph.tep_b = b->ph.surface = 0.0;
    b->ph.source = opts->material.alpha0 != 0.0;
    b->ph.cooling = opts->material.alpha0 * der.l0 * opts->material.g / opts->material.cp;
    b->inst.resize(count);
    for (int i = 0; i < count; ++i) {
        if (meshes[i].nx < 2 || meshes[i].ny < 2) { set_error("instance %d: at least 2x2 cells", i); mp_batch_destroy(b); return MP_ERR_ARG_SIZ; }
        if (mesh_too_large(meshes[i].nx, meshes[i].ny)) { set_error("instance %d: mesh has 2^31 edges or more", i); mp_batch_destroy(b); return MP_ERR_ARG_SIZ; }
        const mp_status s = alloc_instance(b, b->inst[i], meshes[i]);
        if (s != MP_OK) { mp_batch_destroy(b); return s; }
    }
    *out = b;
    return MP_OK;
}

extern "C" void mp_batch_destroy(mp_batch* b) {
    if (!b) return;
    cudaStreamSynchronize(b->stream);
    mp::release_graph(b);
    for (void* p : {(void*)b->d_ctl, (void*)b->d_hdr, (void*)b->d_rep, (void*)b->d_commit}) if (p) cudaFreeAsync(p, b->stream);
    for (void* p : {(void*)b->h_ctl, (void*)b->h_hdr, (void*)b->h_rep}) if (p) cudaFreeHost(p);
    for (MPInstance& in : b->inst) {
        if (in.used && in.arena) cudaFreeAsync(in.arena, b->stream);
        if (in.used && in.src_arena) cudaFreeAsync(in.src_arena, b->stream);
    }
    for (int k = 0; k < mp::NKIND; ++k) if (b->d_args[k]) cudaFreeAsync(b->d_args[k], b->stream);
    for (int k = 0; k < mp::NKIND; ++k) if (b->d_qargs[k]) cudaFreeAsync(b->d_qargs[k], b->stream);
    for (void* p : {(void*)b->d_wqrec, (void*)b->d_wqphase, (void*)b->d_wqface}) if (p) cudaFreeAsync(p, b->stream);
    for (void* p : {(void*)b->d_axpy, (void*)b->d_wrecon, (void*)b->d_wphase, (void*)b->d_wface, (void*)b->d_wsum,
                    (void*)b->d_active, (void*)b->d_part_off, (void*)b->d_part_cnt, (void*)b->d_partial,
                    (void*)b->d_tot, (void*)b->d_status, (void*)b->d_dt})
        if (p) cudaFreeAsync(p, b->stream);
    cudaStreamSynchronize(b->stream);
    for (MPInstance& in : b->inst) if (in.used && in.qbuf) cudaFree(in.qbuf);
    if (b->h_tot) cudaFreeHost(b->h_tot);
    if (b->h_status) cudaFreeHost(b->h_status);
    if (b->h_dt) cudaFreeHost(b->h_dt);
    if (b->h_active) cudaFreeHost(b->h_active);
    for (cudaEvent_t e : b->ev_pool) cudaEventDestroy(e);
    delete b;
}

static mp_status batch_slot(mp_batch* b, int i, MPInstance** out) {
    if (!b) { mp::set_error("null argument"); return MP_ERR_ARG_WRONG; }
    if (i < 0 || i >= (int)b->inst.size() || !b->inst[i].used) { mp::set_error("no instance %d", i); return MP_ERR_ARG_OUTOFRANGE; }
    *out = &b->inst[i];
    return MP_OK;
}

extern "C" mp_status mp_batch_add(mp_batch* b, const mp_mesh_desc* mesh, int* instance) {
    if (!b || !mesh || !instance) { mp::set_error("null argument"); return MP_ERR_ARG_WRONG; }
    if (mesh->nx < 2 || mesh->ny < 2) { mp::set_error("Transport requires at least 2x2 cells"); return MP_ERR_ARG_SIZ; }
    if (mp::mesh_too_large(mesh->nx, mesh->ny)) { mp::set_error("mesh has 2^31 edges or more"); return MP_ERR_ARG_SIZ; }
    int slot = -1;
    for (int i = 0; i < (int)b->inst.size(); ++i) if (!b->inst[i].used) { slot = i; break; }
    if (slot < 0) { slot = (int)b->inst.size(); b->inst.emplace_back(); }
    MP_TRY(mp::alloc_instance(b, b->inst[slot], *mesh));
    *instance = slot;
    return MP_OK;
}

extern "C" mp_status mp_batch_add_quads(mp_batch* b, const mp_mesh_desc* mesh, const double* xy, int* instance) {
    if (!b || !mesh || !xy || !instance) { mp::set_error("null argument"); return MP_ERR_ARG_WRONG; }
    if (mesh->nx < 2 || mesh->ny < 2) { mp::set_error("Transport requires at least 2x2 cells"); return MP_ERR_ARG_SIZ; }
    if (mp::mesh_too_large(mesh->nx, mesh->ny)) { mp::set_error("mesh has 2^31 edges or more"); return MP_ERR_ARG_SIZ; }
    int slot = -1;
    for (int i = 0; i < (int)b->inst.size(); ++i) if (!b->inst[i].used) { slot = i; break; }
    if (slot < 0) { slot = (int)b->inst.size(); b->inst.emplace_back(); }
    const mp_status st = mp::alloc_quad_instance(b, b->inst[slot], *mesh, xy);
    if (st != MP_OK) {
        if (slot == (int)b->inst.size() - 1 && !b->inst[slot].used) b->inst.pop_back();
        return st;
    }
    *instance = slot;
    return MP_OK;
}

extern "C" mp_status mp_batch_remove(mp_batch* b, int i) {
    MPInstance* in;
    MP_TRY(batch_slot(b, i, &in));
    mp::free_instance(b, *in);
    return MP_OK;
}

extern "C" size_t mp_batch_instance_bytes(const mp_mesh_desc* mesh) {
    return mesh ? mp::instance_bytes(mesh->nx, mesh->ny) : 0;
}

extern "C" mp_status mp_batch_set_face_velocity(mp_batch* b, int i, const double* vs_n, const double* ud_n) {
    MPInstance* in;
    MP_TRY(batch_slot(b, i, &in));
    if (!vs_n || !ud_n) { mp::set_error("null argument"); return MP_ERR_ARG_WRONG; }
    MP_CUDA(cudaMemcpyAsync(in->vsn, vs_n, in->NE * mp::kNQ * sizeof(double), cudaMemcpyDefault, b->stream));
    MP_CUDA(cudaMemcpyAsync(in->udn, ud_n, in->NE * mp::kNQ * sizeof(double), cudaMemcpyDefault, b->stream));
    MP_CUDA(cudaStreamSynchronize(b->stream));
    in->have_L = false;
    return MP_OK;
}

extern "C" mp_status mp_batch_set_state(mp_batch* b, int i, const double* H, const double* C, double time) {
    MPInstance* in;
    MP_TRY(batch_slot(b, i, &in));
    if (!H || !C) { mp::set_error("null argument"); return MP_ERR_ARG_WRONG; }
    MP_CUDA(cudaMemcpyAsync(in->H, H, in->N * sizeof(double), cudaMemcpyDefault, b->stream));
    MP_CUDA(cudaMemcpyAsync(in->C, C, in->N * sizeof(double), cudaMemcpyDefault, b->stream));
    MP_CUDA(cudaStreamSynchronize(b->stream));
    in->time = time; in->accepted = 0; in->have_L = false; in->status = 0;
    return MP_OK;
}

extern "C" mp_status mp_batch_get_state(mp_batch* b, int i, double* H, double* C, double* T, double* phi,
                                        double* time, int* accepted, int* status) {
    MPInstance* in;
    MP_TRY(batch_slot(b, i, &in));
    const size_t by = in->N * sizeof(double);
    if (H) MP_CUDA(cudaMemcpyAsync(H, in->H, by, cudaMemcpyDefault, b->stream));
    if (C) MP_CUDA(cudaMemcpyAsync(C, in->C, by, cudaMemcpyDefault, b->stream));
    if (T) MP_CUDA(cudaMemcpyAsync(T, in->T, by, cudaMemcpyDefault, b->stream));
    if (phi) MP_CUDA(cudaMemcpyAsync(phi, in->phi, by, cudaMemcpyDefault, b->stream));
    // time, accepted and status are host records, current once a step call
    // has returned: no wait unless an array was requested.
    if (H || C || T || phi) MP_CUDA(cudaStreamSynchronize(b->stream));
    if (time) *time = in->time;
    if (accepted) *accepted = in->accepted;
    if (status) *status = in->status;
    return MP_OK;
}

extern "C" mp_status mp_batch_step(mp_batch* b, int nsteps, mp_step_report* reports) {
    if (!b) { mp::set_error("null argument"); return MP_ERR_ARG_WRONG; }
    if (nsteps < 0) { mp::set_error("nsteps must be nonnegative"); return MP_ERR_ARG_OUTOFRANGE; }
    bool any = false;
    for (const MPInstance& in : b->inst) any = any || in.used;
    if (b->use_graph && !b->profile && any && nsteps > 0) return mp::graph_steps(b, nsteps, reports);
    std::vector<mp_step_report> reps;
    const int slots = (int)b->inst.size();
    for (int k = 0; k < nsteps; ++k) {
        MP_TRY(mp::step_all(b, reps));
        if (reports)
            for (int i = 0; i < slots; ++i) reports[(size_t)k * slots + i] = reps[i];
    }
    return MP_OK;
}

extern "C" int mp_batch_slots(const mp_batch* b) { return b ? (int)b->inst.size() : 0; }

extern "C" mp_status mp_batch_set_end_time(mp_batch* b, int i, double t_end) {
    MPInstance* in;
    MP_TRY(batch_slot(b, i, &in));
    if (std::isnan(t_end)) { mp::set_error("end time must not be NaN"); return MP_ERR_ARG_OUTOFRANGE; }
    in->t_end = t_end;
    return MP_OK;
}

extern "C" int mp_batch_finished(const mp_batch* b, int i) {
    if (!b || i < 0 || i >= (int)b->inst.size() || !b->inst[i].used) return 0;
    return finished(b->inst[i]) ? 1 : 0;
}

extern "C" size_t mp_batch_bytes_in_use(const mp_batch* b) { return b ? b->bytes_in_use : 0; }

extern "C" mp_status mp_batch_autotune(mp_batch* b, int reps, int* tile, double* best_ms) {
    if (!b) { mp::set_error("null argument"); return MP_ERR_ARG_WRONG; }
    MP_TRY(mp::autotune(b, reps > 0 ? reps : 2, best_ms));
    if (tile) { tile[0] = b->tune.bx; tile[1] = b->tune.by; tile[2] = b->tune.cpt; }
    return MP_OK;
}

extern "C" mp_status mp_batch_profile(mp_batch* b, int enable) {
    if (!b) { mp::set_error("null argument"); return MP_ERR_ARG_WRONG; }
    MP_CUDA(cudaStreamSynchronize(b->stream));
    mp::harvest(b);
    b->profile = enable != 0;
    for (int k = 0; k < 6; ++k) { b->kern_ms[k] = 0; b->kern_n[k] = 0; }
    return MP_OK;
}

extern "C" mp_status mp_batch_kernel_times(mp_batch* b, double ms[6], unsigned long long launches[6]) {
    if (!b || !ms || !launches) { mp::set_error("null argument"); return MP_ERR_ARG_WRONG; }
    MP_CUDA(cudaStreamSynchronize(b->stream));
    mp::harvest(b);
    for (int k = 0; k < 6; ++k) { ms[k] = b->kern_ms[k]; launches[k] = b->kern_n[k]; }
    return MP_OK;
}

extern "C" mp_status mp_batch_set_thermal_bc(mp_batch* b, const int* type, const double* value) {
    if (!b || !type || !value) { mp::set_error("null argument"); return MP_ERR_ARG_WRONG; }
    for (int w = 0; w < 4; ++w) {
        if (type[w] < MP_THERMAL_ZERO_FLUX || type[w] > MP_THERMAL_FLUX) { mp::set_error("unknown thermal condition %d", type[w]); return MP_ERR_ARG_WRONG; }
        if (type[w] != MP_THERMAL_ZERO_FLUX && !std::isfinite(value[w])) { mp::set_error("Boundary data must be finite"); return MP_ERR_ARG_OUTOFRANGE; }
    }
    bool flux = false;
    for (int w = 0; w < 4; ++w) {
        b->ph.wall_type[w] = type[w];
        b->ph.wall_value[w] = type[w] == MP_THERMAL_ZERO_FLUX ? 0.0 : value[w];
        flux = flux || type[w] == MP_THERMAL_FLUX;
    }
    b->ph.diffusion = b->ph.kappa > 0.0 || flux;
    for (auto& in : b->inst) in.have_L = false;
    b->gen += 1;      // the stage kernels take the physics by value
    return MP_OK;
}

extern "C" mp_status mp_batch_set_device_steps(mp_batch* b, int enable) {
    if (!b) { mp::set_error("null argument"); return MP_ERR_ARG_WRONG; }
    b->use_graph = enable != 0;
    return MP_OK;
}

extern "C" mp_status mp_batch_run_stats(const mp_batch* b, unsigned long long* host_syncs,
                                        unsigned long long* graph_captures) {
    if (!b) { mp::set_error("null argument"); return MP_ERR_ARG_WRONG; }
    if (host_syncs) *host_syncs = b->host_syncs;
    if (graph_captures) *graph_captures = b->captures;
    return MP_OK;
}

extern "C" mp_status mp_batch_set_cell_velocity(mp_batch* b, int i, const double* vs_y, const double* ud_y) {
    MPInstance* in;
    MP_TRY(batch_slot(b, i, &in));
    if (!vs_y || !ud_y) { mp::set_error("null argument"); return MP_ERR_ARG_WRONG; }
    const size_t n = in->N * mp::kNQ * mp::kNQ;
    cudaStream_t s = b->stream;
    if (!in->src_arena) {
        const size_t a = (n * sizeof(double) + 255) / 256 * 256, c = (in->N * sizeof(double) + 255) / 256 * 256;
        in->src_bytes = 2 * a + 3 * c;
        MP_CUDA(cudaMallocAsync(&in->src_arena, in->src_bytes, s));
        unsigned char* p = static_cast<unsigned char*>(in->src_arena);
        in->cvs_y = reinterpret_cast<double*>(p); p += a;
        in->cud_y = reinterpret_cast<double*>(p); p += a;
        in->srcH = reinterpret_cast<double*>(p); p += c;
        in->srcR = reinterpret_cast<double*>(p); p += c;
        in->srcS = reinterpret_cast<double*>(p);
        b->bytes_in_use += in->src_bytes;
        b->dirty = true;                // the argument records take the new pointers
    }
    MP_CUDA(cudaMemcpyAsync(in->cvs_y, vs_y, n * sizeof(double), cudaMemcpyDefault, s));
    MP_CUDA(cudaMemcpyAsync(in->cud_y, ud_y, n * sizeof(double), cudaMemcpyDefault, s));
    MP_CUDA(cudaMemsetAsync(in->srcH, 0, 3 * ((in->N * sizeof(double) + 255) / 256 * 256), s));
    MP_CUDA(cudaStreamSynchronize(s));
    in->have_L = false;
    return MP_OK;
}
