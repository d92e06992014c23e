// Stage evaluation that allocates nothing: mp_transport_rhs_noalloc.
//
// Some callers cannot call cudaMalloc: code running inside a host framework
// that owns all device memory through its own pool (and forbids or cannot
// reach the CUDA allocator), or code whose every allocation must happen
// before a latency-critical phase. For them this entry point evaluates one
// transport stage with every piece of scratch memory (per-cell
// reconstruction records, face fluxes, reduction partials, status word)
// taken from one file-scope device array of fixed size; the stencil tables
// travel as kernel parameters. The caller
// still provides the inputs and outputs (device memory).
//
// Limits and behaviour:
//  - at most kMaxCells cells (nx*ny <= 32768); larger meshes are rejected
//    with MP_ERR_ARG_SIZ; the array holds about 7.3 MB on every GPU that
//    loads this library, until the process exits;
//  - every call looks up the array's device address on the current device
//    (cudaGetSymbolAddress, a host-side lookup with no device work), so a
//    context that was torn down and created again is served at its new
//    address;
//  - the call is synchronous: it reads the stage totals and the status word
//    back to the host and waits for the stream;
//  - all calls share the array, and each call overwrites what the previous
//    one left there; calls whose work overlaps on the GPU race on it, so
//    issue them in one stream or serialise them.
#include "common.hpp"
#include "tables.hpp"

namespace mp {

mp_status stage_rhs_raw(int nx, int ny, const mp_transport_opts& o, const double* H, const double* C,
                        const double* vsn, const double* udn, double* rhsH, double* rhsC, double* T, double* phi,
                        double* rate, const StageTables& tab, double* rec, unsigned char* wet, double* face, void* partial,
                        void* totals, unsigned long long* status, mp_stage_totals* out, cudaStream_t s);
size_t raw_partial_bytes(size_t ncell);
size_t raw_totals_bytes();
mp_status validate_opts(const mp_transport_opts& o, mp_derived* der_out);

namespace {

constexpr size_t kMaxCells = 32768;
// nedges = 2*ncells + nx + ny <= 2.5*ncells + 2 for nx, ny >= 2.
constexpr size_t kMaxEdges = kMaxCells * 5 / 2 + 2;
constexpr size_t align256(size_t b) { return (b + 255) / 256 * 256; }
constexpr size_t kRecOff = 0;
constexpr size_t kWetOff = kRecOff + align256(18 * sizeof(double) * kMaxCells);
constexpr size_t kFaceOff = kWetOff + align256(kMaxCells);
constexpr size_t kPartOff = kFaceOff + align256(4 * sizeof(double) * kMaxEdges);
constexpr size_t kPartBytes = align256(((kMaxCells + 255) / 256) * 128);   // >= raw_partial_bytes(kMaxCells)
constexpr size_t kTotOff = kPartOff + kPartBytes;
constexpr size_t kStatOff = kTotOff + 256;
constexpr size_t kScratchBytes = kStatOff + 256;

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

// The device address of g_scratch in the current context. In host code the
// array's name is only a host-side stand-in; kernels need this address.
mp_status scratch_address(unsigned char** out) {
    void* p = nullptr;
    MP_CUDA(cudaGetSymbolAddress(&p, g_scratch));
    *out = static_cast<unsigned char*>(p);
    return MP_OK;
}

}  // namespace
}  // namespace mp

extern "C" mp_status mp_transport_rhs_noalloc(const mp_mesh_desc* mesh, const mp_transport_opts* opts,
                                              const double* H, const double* C, const double* vs_n,
                                              const double* ud_n, double* rhsH, double* rhsC, double* T,
                                              double* phi, double* rate, mp_stage_totals* totals,
                                              mp_stream_t stream) {
    using namespace mp;
    if (!mesh || !opts || !H || !C || !vs_n || !ud_n || !rhsH || !rhsC || !T || !phi) {
        set_error("null argument");
        return MP_ERR_ARG_WRONG;
    }
    if (mesh->nx < 2 || mesh->ny < 2) { set_error("Transport requires at least 2x2 cells"); return MP_ERR_ARG_SIZ; }
    const size_t N = (size_t)mesh->nx * (size_t)mesh->ny;
    if (N > kMaxCells) {
        set_error("mp_transport_rhs_noalloc: %zu cells exceed its fixed scratch limit of %zu cells", N, kMaxCells);
        return MP_ERR_ARG_SIZ;
    }
    // The same option checks as mp_transport_create, then this entry point's own limits.
    MP_TRY(validate_opts(*opts, nullptr));
    if (opts->diffusivity != 0.0) { set_error("thermal diffusion (kappa > 0) is not supported by mp_transport_rhs_noalloc"); return MP_ERR_ARG_WRONG; }
    if (opts->material.alpha0 != 0.0) { set_error("adiabatic source (alpha0 != 0) is not supported by mp_transport_rhs_noalloc"); return MP_ERR_ARG_WRONG; }
    if (opts->precision != MP_PRECISION_FP64) { set_error("mp_transport_rhs_noalloc evaluates the FP64 stage"); return MP_ERR_ARG_WRONG; }
    if (raw_partial_bytes(N) > kPartBytes || raw_totals_bytes() > 256) { set_error("scratch layout too small"); return MP_ERR_ARG_SIZ; }
    StageTables tab;
    const int tb = build_stage_tables(mesh->nx, mesh->ny, mesh->x0, mesh->x1, mesh->y0, mesh->y1, tab);
    if (tb) { set_error("stencil table construction failed"); return (mp_status)tb; }
    unsigned char* base = nullptr;
    MP_TRY(scratch_address(&base));
    cudaStream_t s = (cudaStream_t)stream;
    return stage_rhs_raw(mesh->nx, mesh->ny, *opts, H, C, vs_n, ud_n, rhsH, rhsC, T, phi, rate, tab,
                         reinterpret_cast<double*>(base + kRecOff), base + kWetOff,
                         reinterpret_cast<double*>(base + kFaceOff), base + kPartOff, base + kTotOff,
                         reinterpret_cast<unsigned long long*>(base + kStatOff), totals, s);
}
