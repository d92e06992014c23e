// Device-side control of the coupled SSP Runge-Kutta time step, one record
// per instance, so a run of many steps needs no host round trip between
// stages.
//
// The rule is the reference's Run loop (src/couple/evolve.cpp:449-507): dt =
// min(remaining, cap, cfl / rate of L(U^n)) (the "fixed" control keeps dt =
// min(remaining, dt_initial) and fails when that exceeds the CFL bound,
// :456,483); stage 1 admissibility; per later stage the status word, a finite
// rate, courant = dt * max(stage rates) <= cfl (1 + 1e-12) and admissibility
// of the combined state; halve and retry (<= 40, dt >= min(remaining,
// dt_min)); the balance check (:486-490); commit; L(U^{n+1}). Every decision
// is a short sequence of explicitly rounded FP64 operations (no contraction),
// the same operations in the same order as the host-driven loops, so a run
// controlled here takes the same dt, retries and results bit for bit.
//
// The control kernels run as one block over all instances between the stage
// kernels of a CUDA graph; they set the `active` gate each stage kernel reads,
// the device dt the RK kernels read, and the graph's loop conditions. Every
// loop they drive is bounded by a counter: at most kMaxAttempts attempts per
// step, and the caller's step count.
#ifndef MP_STEP_CTL_CUH
#define MP_STEP_CTL_CUH

#include "common.hpp"
#include "stage_kernels.cuh"

namespace mp {
namespace {

constexpr int kMaxAttempts = 41;     // the first attempt and 40 retries
constexpr int kCtlThreads = 256;

// Options of the step rule (per run, identical for every instance).
struct StepOpts {
    double cfl, dt_initial, dt_max, dt_min, Xe;
    int rk3;            // Shu-Osher SSPRK3 (else SSPRK2)
    int fixed;          // "fixed" time control
    // Conventions of the calling API:
    int snap_end;       // after a step within 32 eps of t_end, time = t_end (batched engine)
    int end_reports;    // a step not taken at the end time reports time = t_end (single instance)
    int restore_time;   // a failure after commit restores the step's start time (single instance)
};

// Why an instance's step failed, for the host's message.
enum : int {
    FAIL_NONE = 0, FAIL_STAGE = 1, FAIL_RATE = 2, FAIL_RETRIES = 3, FAIL_FIXED_LIMIT = 4, FAIL_FIXED_STAGE = 5,
    FAIL_BALANCE = 6
};

struct InstCtl {
    // Persistent state of the instance (mirrored on the host between runs).
    double time, t_end;
    int used, accepted, status, have_L;
    int fail, fail_stage;             // FAIL_* and the stage (2, 3, or 4 for L(U^{n+1}))
    unsigned long long word;          // status word of a failing stage
    double bal_H, bal_C;              // balance errors of a failed balance check
    Totals cur;                       // totals of L(U^n)
    // The step in progress.
    double dt, start, remaining, courant;
    int retries, pending, valid, done;
    Totals first, second, third;
};

struct CtlHeader {
    int step, nsteps;                 // steps taken in this launch / requested
    int attempts;                     // attempts of the current step
    int total_attempts;               // over the launch (kernel count)
    int stop;                         // a single instance failed: no further steps
};

// Explicitly rounded FP64 (the host loops compile without contraction).
__device__ __forceinline__ double ad(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sb(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double ml(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dv(double a, double b) { return __ddiv_rn(a, b); }
// std::min / std::max as the host evaluates them.
__device__ __forceinline__ double mn(double a, double b) { return b < a ? b : a; }
__device__ __forceinline__ double mx(double a, double b) { return a < b ? b : a; }

__device__ __forceinline__ bool admissible_dev(const Totals& t, double Xe) {
    return t.nonfinite == 0.0 && t.Hmin >= 0.0 && t.Cmin >= 0.0 && t.Cmax <= Xe;
}

// Within 32 eps of the end time (evolve.cpp:450-451).
__device__ __forceinline__ bool at_end(double time, double t_end) {
    if (!isfinite(t_end)) return false;
    return sb(t_end, time) <= ml(32 * 2.220446049250313e-16, mx(1.0, fabs(t_end)));
}

__device__ __forceinline__ int word_code(unsigned long long w) { return (int)(w & 0xff); }

__device__ __forceinline__ void fail_inst(InstCtl& c, int status, int fail) {
    c.status = status; c.fail = fail; c.pending = 0; c.valid = 0; c.done = 0;
}

// Block-wide "any" of a per-thread flag (one block of kCtlThreads).
__device__ __forceinline__ int block_any(int v) { return __syncthreads_or(v); }

// Start of a step: dt of every healthy instance; the attempt loop's
// condition. reps: this step's report row.
__global__ void __launch_bounds__(kCtlThreads) ctl_begin_kernel(InstCtl* ctl, int n, StepOpts so, CtlHeader* hdr,
                                                                mp_step_report* reps, cudaGraphConditionalHandle attempt) {
    int any = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        InstCtl& c = ctl[i];
        mp_step_report& r = reps[(size_t)hdr->step * n + i];
        r = mp_step_report{};
        c.pending = c.valid = c.done = 0;
        if (!c.used || c.status || hdr->stop) { r.status = c.status; continue; }
        if (at_end(c.time, c.t_end)) {
            c.time = c.t_end;
            if (so.end_reports) r.time = c.t_end;
            continue;
        }
        c.first = c.cur;
        c.remaining = sb(c.t_end, c.time);
        const double cap = so.fixed ? so.dt_initial : (c.accepted == 0 ? so.dt_initial : so.dt_max);
        const double limit = c.cur.maxRate > 0 ? dv(so.cfl, c.cur.maxRate) : so.dt_max;
        double dt = mn(c.remaining, cap);
        if (so.fixed && !(dt <= ml(limit, 1 + 1e-12))) { fail_inst(c, MP_ERR_ARG_OUTOFRANGE, FAIL_FIXED_LIMIT); r.status = c.status; continue; }
        if (!so.fixed) dt = mn(dt, limit);
        c.dt = dt;
        c.start = c.time;
        c.retries = 0;
        c.courant = 0.0;
        c.pending = 1;
        any = 1;
    }
    any = block_any(any);
    if (threadIdx.x == 0) {
        hdr->attempts = 0;
        cudaGraphSetConditional(attempt, any ? 1u : 0u);
    }
}

// Start of an attempt: the retry bounds, the stage-1 gate and the device dt.
__global__ void __launch_bounds__(kCtlThreads) ctl_attempt_kernel(InstCtl* ctl, int n, StepOpts so, CtlHeader* hdr,
                                                                  int* active, double* dt_dev) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        InstCtl& c = ctl[i];
        if (c.pending && !(c.dt >= mn(c.remaining, so.dt_min) && c.retries < 40))
            fail_inst(c, MP_ERR_NOT_CONVERGED, FAIL_RETRIES);
        active[i] = c.pending;
        if (c.pending) dt_dev[i] = c.dt;
    }
    if (threadIdx.x == 0) { hdr->attempts += 1; hdr->total_attempts += 1; }
}

// After U1 = U^n + dt L^n: admissibility of U1 gates the next stage.
__global__ void __launch_bounds__(kCtlThreads) ctl_after_axpy_kernel(InstCtl* ctl, int n, StepOpts so, const Totals* tot,
                                                                     unsigned long long* words, int* active) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        InstCtl& c = ctl[i];
        c.valid = c.pending && admissible_dev(tot[i], so.Xe);
        active[i] = c.valid;
        words[i] = ~0ULL;
    }
}

// After stage `which` (2 or 3) of an attempt. `last`: the attempt ends here
// (accept, fail, or halve dt and set the loop condition for a retry).
__global__ void __launch_bounds__(kCtlThreads) ctl_after_stage_kernel(InstCtl* ctl, int n, StepOpts so, const Totals* tot,
                                                                      unsigned long long* words, int* active, int which,
                                                                      int last, CtlHeader* hdr,
                                                                      cudaGraphConditionalHandle attempt) {
    int any = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        InstCtl& c = ctl[i];
        if (c.valid) {
            const unsigned long long w = words[i];
            if (w != ~0ULL) {
                fail_inst(c, word_code(w), FAIL_STAGE);
                c.word = w; c.fail_stage = which;
            } else if (!isfinite(tot[i].maxRate)) {
                fail_inst(c, MP_ERR_FP, FAIL_RATE);
                c.fail_stage = which;
            } else {
                const Totals& t = tot[i];
                double rate = mx(c.first.maxRate, t.maxRate);
                if (which == 2) c.second = t;
                else { c.third = t; rate = mx(mx(c.first.maxRate, c.second.maxRate), t.maxRate); }
                c.courant = ml(c.dt, rate);
                c.valid = c.courant <= ml(so.cfl, 1 + 1e-12) && admissible_dev(t, so.Xe);
            }
        }
        words[i] = ~0ULL;
        if (last && c.pending) {
            if (c.valid) { c.done = 1; c.pending = 0; }
            else if (so.fixed) fail_inst(c, MP_ERR_ARG_OUTOFRANGE, FAIL_FIXED_STAGE);
            else { c.dt = ml(c.dt, 0.5); c.retries += 1; }
        }
        active[i] = c.valid;
        any |= c.pending;
    }
    if (last) {
        any = block_any(any);
        if (any && hdr->attempts >= kMaxAttempts) {
            // Unreachable by the retry rule above (40 retries fail in the
            // next attempt); a hard stop for the graph's attempt loop.
            for (int i = threadIdx.x; i < n; i += blockDim.x)
                if (ctl[i].pending) fail_inst(ctl[i], MP_ERR_NOT_CONVERGED, FAIL_RETRIES);
            any = 0;
        }
        if (threadIdx.x == 0) cudaGraphSetConditional(attempt, any ? 1u : 0u);
    }
}

// Balance check (evolve.cpp:486-490), commit bookkeeping and the report;
// `active` gates the state copy and the evaluation of L(U^{n+1}).
__global__ void __launch_bounds__(kCtlThreads) ctl_commit_kernel(InstCtl* ctl, int n, StepOpts so, CtlHeader* hdr,
                                                                 mp_step_report* reps, unsigned long long* words,
                                                                 int* active) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        InstCtl& c = ctl[i];
        words[i] = ~0ULL;
        if (c.done) {
            const Totals& f = c.first;
            const Totals& s = c.second;
            const Totals& fin = so.rk3 ? c.third : c.second;
            double repH, repC, repS, bH, bC;
            if (so.rk3) {
                const double two3 = 2.0 / 3.0;
                repH = ad(dv(ad(f.bH, s.bH), 6.0), ml(c.third.bH, two3));
                repC = ad(dv(ad(f.bC, s.bC), 6.0), ml(c.third.bC, two3));
                repS = ad(dv(ad(f.sH, s.sH), 6.0), ml(c.third.sH, two3));
                bH = ad(sb(fin.HI, f.HI), ml(c.dt, sb(repH, repS)));
                bC = ad(sb(fin.CI, f.CI), ml(c.dt, repC));
            } else {
                repH = ml(.5, ad(f.bH, s.bH));
                repC = ml(.5, ad(f.bC, s.bC));
                repS = ml(.5, ad(f.sH, s.sH));
                bH = ad(sb(fin.HI, f.HI), ml(ml(.5, c.dt), sb(sb(ad(f.bH, s.bH), f.sH), s.sH)));
                bC = ad(sb(fin.CI, f.CI), ml(ml(.5, c.dt), ad(f.bC, s.bC)));
            }
            if (!(fabs(bH) < ml(1e-10, mx(1.0, fabs(f.HI))) && fabs(bC) < 1e-10)) {
                fail_inst(c, MP_ERR_PLIB, FAIL_BALANCE);
                c.bal_H = bH; c.bal_C = bC;
            } else {
                c.time = ad(c.start, c.dt);
                if (so.snap_end && at_end(c.time, c.t_end)) c.time = c.t_end;
                c.have_L = 0;
                mp_step_report& r = reps[(size_t)hdr->step * n + i];
                r.retries = c.retries; r.dt = c.dt; r.time = c.time; r.courant = c.courant;
                r.boundaryH = repH; r.boundaryC = repC; r.sourceH = repS;
                r.balanceH = bH; r.balanceC = bC; r.H_integral = fin.HI; r.C_integral = fin.CI;
            }
        }
        active[i] = c.done;
    }
}

// After L(U^{n+1}): the new L's totals, the step count and the run's loop
// condition (bounded by the requested step count).
__global__ void __launch_bounds__(kCtlThreads) ctl_after_rhs_kernel(InstCtl* ctl, int n, StepOpts so, const Totals* tot,
                                                                    unsigned long long* words, mp_step_report* reps,
                                                                    CtlHeader* hdr, int stop_on_fail,
                                                                    cudaGraphConditionalHandle run) {
    int failed = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        InstCtl& c = ctl[i];
        mp_step_report& r = reps[(size_t)hdr->step * n + i];
        if (c.done) {
            const unsigned long long w = words[i];
            if (w != ~0ULL) { fail_inst(c, word_code(w), FAIL_STAGE); c.word = w; c.fail_stage = 4; }
            else if (!isfinite(tot[i].maxRate)) { fail_inst(c, MP_ERR_FP, FAIL_RATE); c.fail_stage = 4; }
            if (c.status) {
                if (so.restore_time) c.time = c.start;
            } else {
                c.cur = tot[i];
                c.have_L = 1;
                c.accepted += 1;
                r.maxRate = c.cur.maxRate;
                r.divergence = c.cur.divergence;
            }
        }
        words[i] = ~0ULL;
        if (c.used) r.status = c.status;
        failed |= c.used && c.status != 0;
        c.done = 0;
    }
    failed = block_any(failed);
    if (threadIdx.x == 0) {
        if (stop_on_fail && failed) hdr->stop = 1;
        hdr->step += 1;
        const bool more = hdr->step < hdr->nsteps && !hdr->stop;
        cudaGraphSetConditional(run, more ? 1u : 0u);
    }
}

}  // namespace
}  // namespace mp

#endif
