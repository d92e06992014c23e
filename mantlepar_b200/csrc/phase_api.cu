// Phase-equilibrium entry points of the C ABI and the batched FP64 kernel.
//
// mp_phase_* replace mantle::phase::EutecticModel
// (src/phase/eutectic_rescaled.h:103-136): parameters are validated and the
// scales derived on the host exactly as the reference's derive()
// (eutectic_rescaled.cpp:42-86, long double intermediates), the pointwise
// inversion runs on the GPU.
#include "common.hpp"
#include "phase_math.cuh"

#include <cmath>
#include <cstring>
#include <limits>
#include <mutex>
#include <string>

namespace mp {

std::atomic<unsigned long long> g_launches{0};

static thread_local std::string g_error;

void set_error(const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_error = buf;
}

namespace {

typedef long double ld;

struct DeriveFail { mp_status code; const char* what; };

double checked(ld v, const char* what) {
    if (!std::isfinite(v) || std::fabs(v) > (ld)std::numeric_limits<double>::max()) throw DeriveFail{MP_ERR_PHASE_OVERFLOW, what};
    return (double)v;
}
double positive_scale(ld v, const char* what) {
    const double r = checked(v, what);
    if (r <= 0.0) throw DeriveFail{MP_ERR_PHASE_OVERFLOW, what};
    return r;
}
void need_finite(double v, const char* what) { if (!std::isfinite(v)) throw DeriveFail{MP_ERR_PHASE_INVALID, what}; }
void need_positive(double v, const char* what) { need_finite(v, what); if (v <= 0.0) throw DeriveFail{MP_ERR_PHASE_INVALID, what}; }

// Parameter validation and scales (eutectic_rescaled.cpp:42-86).
mp_derived derive(const mp_material& p) {
    need_positive(p.Tm0, "Tm0 must be positive");
    need_positive(p.Te0, "Te0 must be positive");
    if (p.Tm0 <= p.Te0) throw DeriveFail{MP_ERR_PHASE_INVALID, "Tm0 must be greater than Te0"};
    need_finite(p.nu, "nu must be finite");
    if (p.nu == 0.0) throw DeriveFail{MP_ERR_PHASE_INVALID, "nu must be nonzero"};
    need_positive(p.L, "L must be positive");
    need_positive(p.cp, "cp must be positive");
    need_finite(p.Xe, "Xe must be finite");
    if (p.Xe <= 0.0 || p.Xe >= 1.0) throw DeriveFail{MP_ERR_PHASE_INVALID, "Xe must lie strictly between 0 and 1"};
    need_positive(p.rho, "rho must be positive");
    need_positive(p.rhor, "rhor must be positive");
    need_positive(p.mus, "mus must be positive");
    need_positive(p.mul, "mul must be positive");
    need_positive(p.k0, "k0 must be positive");
    need_positive(p.g, "g must be positive");
    need_finite(p.alpha0, "alpha0 must be finite");
    mp_derived d{};
    const ld span = (ld)p.Tm0 - p.Te0;
    const ld h0 = (ld)p.cp * span;
    d.dT = positive_scale(span, "dT is not a positive scale");
    d.h0 = positive_scale(h0, "h0 is not a positive scale");
    d.gamma = checked(1.0L / p.nu, "gamma is not representable");
    if (d.gamma == 0.0) throw DeriveFail{MP_ERR_PHASE_OVERFLOW, "gamma underflows to zero"};
    d.LD = positive_scale(p.L / h0, "LD is not a positive scale");
    d.TDm0 = positive_scale(p.Tm0 / span, "TDm0 is not a positive scale");
    d.TDe0 = positive_scale(p.Te0 / span, "TDe0 is not a positive scale");
    d.invk0 = positive_scale(1.0L / p.k0, "invk0 is not a positive scale");
    const ld l0 = std::sqrt((ld)p.mus * p.k0 / p.mul);
    const ld u0 = (ld)p.k0 * p.rhor * p.g / p.mul;
    d.l0 = positive_scale(l0, "l0 is not a positive scale");
    d.u0 = positive_scale(u0, "u0 is not a positive scale");
    d.p0 = positive_scale((ld)p.rhor * p.g * l0, "p0 is not a positive scale");
    d.t0 = positive_scale(l0 / u0, "t0 is not a positive scale");
    return d;
}

const char* phase_message(int code) {
    switch (code) {
    case PH_INVALID: return "invalid phase input (non-finite value or C outside [0, Xe])";
    case PH_OVERFLOW: return "phase temperature/enthalpy not representable";
    case PH_RUNTIME: return "computed phase fraction is outside [0, 1]";
    default: return "phase evaluation failed";
    }
}

__global__ void phase_batch_kernel(PhaseConst k, const double* __restrict__ H, const double* __restrict__ C,
                                   const double* __restrict__ P, double P_const, size_t n, mp_phase_soa out,
                                   unsigned long long* __restrict__ first_bad) {
    const double nan = __longlong_as_double(0x7ff8000000000000ULL);
    double Tep0 = 0.0;
    int st0 = P ? PH_OK : eutectic_temperature(k, P_const, Tep0);
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        double Tep = Tep0;
        int st = st0;
        if (P) st = eutectic_temperature(k, P[i], Tep);
        PhaseOut s;
        s.region = 0;   // set by phase_eval once the region is selected
        if (!st) st = phase_eval(k, H[i], C[i], Tep, s);
        if (st) {
            // The region stays when the failure came after its selection.
            s.phi1 = s.phi2 = s.phil = s.cl = s.cs = s.T = s.Tep = s.dTdC = s.dTdH = nan;
            s.flags = 0;
            atomicMin(first_bad, ((unsigned long long)i << 8) | (unsigned long long)st);
        }
        if (out.phi1) out.phi1[i] = s.phi1;
        if (out.phi2) out.phi2[i] = s.phi2;
        if (out.phil) out.phil[i] = s.phil;
        if (out.cl) out.cl[i] = s.cl;
        if (out.cs) out.cs[i] = s.cs;
        if (out.TDp) out.TDp[i] = s.T;
        if (out.Tep) out.Tep[i] = s.Tep;
        if (out.dTD_dCD) out.dTD_dCD[i] = s.dTdC;
        if (out.dTD_dHD) out.dTD_dHD[i] = s.dTdH;
        if (out.region) out.region[i] = (int8_t)s.region;
        if (out.flags) out.flags[i] = (uint8_t)s.flags;
    }
}

}  // namespace

PhaseConst phase_const(const mp_material& p, const mp_derived& d) {
    PhaseConst k;
    k.Xe = p.Xe; k.LD = d.LD; k.sqrtLD = std::sqrt(d.LD); k.TDe0 = d.TDe0; k.nu = p.nu; k.dT = d.dT;
    return k;
}

mp_status derive_checked(const mp_material& p, mp_derived& d) {
    try { d = derive(p); return MP_OK; }
    catch (const DeriveFail& f) { set_error("%s", f.what); return f.code; }
}

}  // namespace mp

struct mp_phase_model {
    mp_material params;
    mp_derived derived;
    mp::PhaseConst k;
    unsigned long long* d_bad = nullptr;   // device word for the first failing index
    unsigned long long* h_bad = nullptr;   // pinned mirror
    // mp_phase_evaluate_host: device staging of host inputs/outputs, grown on
    // demand and serialised per model (evaluate() is const and may be called
    // from several threads).
    std::mutex host_lock;
    unsigned char* d_stage = nullptr;
    size_t stage_bytes = 0;
};

extern "C" const char* mp_last_error_string(void) { return mp::g_error.c_str(); }

extern "C" unsigned long long mp_kernel_launches(void) { return mp::g_launches.load(); }

extern "C" mp_status mp_phase_create(const mp_material* params, mp_phase_model** model) {
    if (!params || !model) { mp::set_error("null argument"); return MP_ERR_ARG_WRONG; }
    mp_derived d;
    MP_TRY(mp::derive_checked(*params, d));
    mp_phase_model* m = new mp_phase_model;
    m->params = *params; m->derived = d; m->k = mp::phase_const(*params, d);
    cudaError_t e = cudaMalloc(&m->d_bad, sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMallocHost(&m->h_bad, sizeof(unsigned long long));
    if (e != cudaSuccess) { mp_phase_destroy(m); return mp::cuda_status(e, "mp_phase_create"); }
    *model = m;
    return MP_OK;
}

extern "C" mp_status mp_phase_set_params(mp_phase_model* m, const mp_material* params) {
    if (!m || !params) { mp::set_error("null argument"); return MP_ERR_ARG_WRONG; }
    mp_derived d;
    MP_TRY(mp::derive_checked(*params, d));   // a rejected update leaves the model unchanged
    m->params = *params; m->derived = d; m->k = mp::phase_const(*params, d);
    return MP_OK;
}

extern "C" mp_status mp_phase_get_params(const mp_phase_model* m, mp_material* params) {
    if (!m || !params) { mp::set_error("null argument"); return MP_ERR_ARG_WRONG; }
    *params = m->params;
    return MP_OK;
}

extern "C" mp_status mp_phase_get_derived(const mp_phase_model* m, mp_derived* d) {
    if (!m || !d) { mp::set_error("null argument"); return MP_ERR_ARG_WRONG; }
    *d = m->derived;
    return MP_OK;
}

extern "C" void mp_phase_destroy(mp_phase_model* m) {
    if (!m) return;
    if (m->d_bad) cudaFree(m->d_bad);
    if (m->h_bad) cudaFreeHost(m->h_bad);
    if (m->d_stage) cudaFree(m->d_stage);
    delete m;
}

extern "C" mp_status mp_phase_boundaries(const mp_phase_model* m, double C, double P, mp_phase_bounds* out) {
    if (!m || !out) { mp::set_error("null argument"); return MP_ERR_ARG_WRONG; }
    double Tep;
    int st = mp::eutectic_temperature(m->k, P, Tep);
    mp::Bounds b;
    if (!st) st = mp::bounds_at(m->k, C, Tep, b);
    if (st) { mp::set_error("%s", st == mp::PH_INVALID ? "CD must lie in [0, Xe] and P must be finite" : "Phase temperature/enthalpy intervals are not resolvable"); return (mp_status)st; }
    out->Tep = b.Tep; out->Tmp = b.Tmp; out->H_eutectic_end = b.Heut; out->H_liquidus = b.Hliq;
    return MP_OK;
}

extern "C" mp_status mp_phase_evaluate_batch(const mp_phase_model* m, const double* H, const double* C,
                                             const double* P, double P_const, size_t n,
                                             const mp_phase_soa* out, long long* first_bad, mp_stream_t stream) {
    if (!m || !out || (n && (!H || !C))) { mp::set_error("null argument"); return MP_ERR_ARG_WRONG; }
    if (first_bad) *first_bad = -1;
    if (n == 0) return MP_OK;
    cudaStream_t s = (cudaStream_t)stream;
    MP_CUDA(cudaMemsetAsync(m->d_bad, 0xff, sizeof(unsigned long long), s));
    int sms = 148;
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int threads = 256;
    size_t blocks = (n + threads - 1) / threads;
    const size_t cap = (size_t)sms * 16;
    if (blocks > cap) blocks = cap;
    mp::phase_batch_kernel<<<(unsigned)blocks, threads, 0, s>>>(m->k, H, C, P, P_const, n, *out, m->d_bad);
    mp::count_launch();
    MP_CUDA(cudaGetLastError());
    MP_CUDA(cudaMemcpyAsync(m->h_bad, m->d_bad, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
    MP_CUDA(cudaStreamSynchronize(s));
    const unsigned long long v = *m->h_bad;
    if (v == ~0ULL) return MP_OK;
    const long long idx = (long long)(v >> 8);
    const int code = (int)(v & 0xff);
    if (first_bad) *first_bad = idx;
    mp::set_error("point %lld: %s", idx, mp::phase_message(code));
    return (mp_status)code;
}

extern "C" mp_status mp_phase_evaluate_host(const mp_phase_model* mc, const double* H, const double* C, const double* P,
                                            double P_const, size_t n, const mp_phase_soa* out, long long* first_bad) {
    if (!mc || !out || (n && (!H || !C))) { mp::set_error("null argument"); return MP_ERR_ARG_WRONG; }
    if (first_bad) *first_bad = -1;
    if (n == 0) return MP_OK;
    mp_phase_model* m = const_cast<mp_phase_model*>(mc);
    std::lock_guard<std::mutex> g(m->host_lock);
    // Staging: H, C, P, then the nine double fields, then region and flags.
    const size_t dbl = n * sizeof(double);
    const size_t need = 12 * dbl + 2 * n;
    if (m->stage_bytes < need) {
        if (m->d_stage) cudaFree(m->d_stage);
        m->d_stage = nullptr;
        m->stage_bytes = 0;
        MP_CUDA(cudaMalloc(&m->d_stage, need));
        m->stage_bytes = need;
    }
    double* dH = reinterpret_cast<double*>(m->d_stage);
    double* dC = dH + n;
    double* dP = dC + n;
    double* fields = dP + n;
    int8_t* dregion = reinterpret_cast<int8_t*>(fields + 9 * n);
    uint8_t* dflags = reinterpret_cast<uint8_t*>(dregion + n);
    MP_CUDA(cudaMemcpy(dH, H, dbl, cudaMemcpyHostToDevice));
    MP_CUDA(cudaMemcpy(dC, C, dbl, cudaMemcpyHostToDevice));
    if (P) MP_CUDA(cudaMemcpy(dP, P, dbl, cudaMemcpyHostToDevice));
    double* const* hsrc[9] = {&out->phi1, &out->phi2, &out->phil, &out->cl, &out->cs,
                              &out->TDp, &out->Tep, &out->dTD_dCD, &out->dTD_dHD};
    mp_phase_soa d{};
    double** dst[9] = {&d.phi1, &d.phi2, &d.phil, &d.cl, &d.cs, &d.TDp, &d.Tep, &d.dTD_dCD, &d.dTD_dHD};
    for (int k = 0; k < 9; ++k) *dst[k] = *hsrc[k] ? fields + k * n : nullptr;
    d.region = out->region ? dregion : nullptr;
    d.flags = out->flags ? dflags : nullptr;
    long long bad = -1;
    const mp_status st = mp_phase_evaluate_batch(m, dH, dC, P ? dP : nullptr, P_const, n, &d, &bad, nullptr);
    if (st != MP_OK && bad < 0) return st;   // launch/runtime failure: nothing was evaluated
    const std::string msg = st != MP_OK ? mp_last_error_string() : std::string();
    for (int k = 0; k < 9; ++k)
        if (*hsrc[k]) MP_CUDA(cudaMemcpy(*hsrc[k], fields + k * n, dbl, cudaMemcpyDeviceToHost));
    if (out->region) MP_CUDA(cudaMemcpy(out->region, dregion, n, cudaMemcpyDeviceToHost));
    if (out->flags) MP_CUDA(cudaMemcpy(out->flags, dflags, n, cudaMemcpyDeviceToHost));
    if (first_bad) *first_bad = bad;
    if (st != MP_OK) mp::set_error("%s", msg.c_str());
    return st;
}

namespace {
// The reference's requireFinite / requirePositive / checkedDouble
// (eutectic_rescaled.cpp:13-32) as status codes.
mp_status need_finite(double v, const char* name) {
    if (std::isfinite(v)) return MP_OK;
    mp::set_error("%s must be finite", name);
    return MP_ERR_PHASE_INVALID;
}
mp_status checked_out(long double v, const char* name, double* out) {
    if (!std::isfinite(v) || std::fabs(v) > (long double)std::numeric_limits<double>::max()) {
        mp::set_error("%s is not representable", name);
        return MP_ERR_PHASE_OVERFLOW;
    }
    *out = (double)v;
    return MP_OK;
}
}  // namespace

extern "C" mp_status mp_phase_pressure_corrected_temperature(const mp_phase_model* m, double TD, double P,
                                                             double* out) {
    if (!m || !out) { mp::set_error("null argument"); return MP_ERR_ARG_WRONG; }
    MP_TRY(need_finite(TD, "TD"));
    MP_TRY(need_finite(P, "P"));
    const long double shift = (long double)P / m->params.nu / m->derived.dT;
    return checked_out((long double)TD + shift, "pressure-corrected temperature", out);
}

extern "C" mp_status mp_phase_static_pressure(const mp_phase_model* m, double zD, double length_scale, double* out) {
    if (!m || !out) { mp::set_error("null argument"); return MP_ERR_ARG_WRONG; }
    MP_TRY(need_finite(zD, "zD"));
    MP_TRY(need_finite(length_scale, "length_scale"));
    if (length_scale <= 0.0) { mp::set_error("length_scale must be positive"); return MP_ERR_PHASE_INVALID; }
    return checked_out((long double)m->params.rho * m->params.g * zD * length_scale, "static pressure", out);
}
