// CPU oracle: restatement of the binary eutectic equilibrium.
// TEST INFRASTRUCTURE ONLY -- the checker for the CUDA phase kernel.
//
// Follows src/phase/eutectic_rescaled.cpp of the reference:
//   derive()            :42-86   scales (long double intermediates)
//   selectRegion()      :95-105  region ownership at the interfaces
//   unitFraction()      :108-114 clip of roundoff excursions, else runtime error
//   boundaries()        :163-185 pressure-corrected interval ends
//   evaluate()          :192-282 closed forms per region
// The intermediate precision (80-bit long double on x86-64) is kept so that
// the restatement reproduces the compiled reference bit for bit.
#include "oracle.h"

#include <algorithm>
#include <cmath>
#include <limits>

namespace {

typedef long double ld;
// Per-cell evaluation type: long double as in the reference; ORC_FP64_CELL
// evaluates the per-cell steps in double (the derived scales stay long double).
#ifdef ORC_FP64_CELL
typedef double lc;
#else
typedef long double lc;
#endif

struct Fail { int code; };

inline void finite_or_throw(double v) { if (!std::isfinite(v)) throw Fail{ORC_INVALID}; }
inline void positive_or_throw(double v) { finite_or_throw(v); if (v <= 0.0) throw Fail{ORC_INVALID}; }

// eutectic_rescaled.cpp:26-32: representable as double, else overflow_error.
inline double to_double_checked(ld v) {
    if (!std::isfinite(v) || std::fabs(v) > (ld)std::numeric_limits<double>::max()) throw Fail{ORC_OVERFLOW};
    return (double)v;
}
inline double positive_scale(ld v) {
    double r = to_double_checked(v);
    if (r <= 0.0) throw Fail{ORC_OVERFLOW};
    return r;
}

// eutectic_rescaled.cpp:42-86
orc_derived derive_or_throw(const orc_material& p) {
    positive_or_throw(p.Tm0);
    positive_or_throw(p.Te0);
    if (p.Tm0 <= p.Te0) throw Fail{ORC_INVALID};
    finite_or_throw(p.nu);
    if (p.nu == 0.0) throw Fail{ORC_INVALID};
    positive_or_throw(p.L);
    positive_or_throw(p.cp);
    finite_or_throw(p.Xe);
    if (p.Xe <= 0.0 || p.Xe >= 1.0) throw Fail{ORC_INVALID};
    positive_or_throw(p.rho); positive_or_throw(p.rhor); positive_or_throw(p.mus);
    positive_or_throw(p.mul); positive_or_throw(p.k0); positive_or_throw(p.g);
    finite_or_throw(p.alpha0);
    orc_derived d{};
    const ld span = (ld)p.Tm0 - p.Te0;
    const ld enthalpy = (ld)p.cp * span;
    d.dT = positive_scale(span);
    d.h0 = positive_scale(enthalpy);
    d.gamma = to_double_checked(1.0L / p.nu);
    if (d.gamma == 0.0) throw Fail{ORC_OVERFLOW};
    d.LD = positive_scale(p.L / enthalpy);
    d.TDm0 = positive_scale(p.Tm0 / span);
    d.TDe0 = positive_scale(p.Te0 / span);
    d.invk0 = positive_scale(1.0L / p.k0);
    const ld length = std::sqrt((ld)p.mus * p.k0 / p.mul);
    const ld velocity = (ld)p.k0 * p.rhor * p.g / p.mul;
    d.l0 = positive_scale(length);
    d.u0 = positive_scale(velocity);
    d.p0 = positive_scale((ld)p.rhor * p.g * length);
    d.t0 = positive_scale(length / velocity);
    return d;
}

// eutectic_rescaled.cpp:143-149 (pressureCorrectedTemperature)
double shifted_temperature(const orc_material& p, const orc_derived& d, double TD, double P) {
    finite_or_throw(TD);
    finite_or_throw(P);
    const lc shift = (lc)P / p.nu / d.dT;
    return to_double_checked((lc)TD + shift);
}

// eutectic_rescaled.cpp:163-185
orc_bounds bounds_or_throw(const orc_material& p, const orc_derived& d, double C, double P) {
    finite_or_throw(C);
    if (C < 0.0 || C > p.Xe) throw Fail{ORC_INVALID};
    orc_bounds b{};
    b.Tep = shifted_temperature(p, d, d.TDe0, P);
    b.Tmp = to_double_checked((lc)b.Tep + 1.0L);
    const lc r = (lc)C / p.Xe;
    b.H_eutectic_end = to_double_checked((lc)b.Tep + d.LD * r);
    b.H_liquidus = to_double_checked((lc)b.Tep + (1.0L - r) + d.LD);
    if (C == 0.0) b.H_liquidus = to_double_checked((lc)b.Tmp + d.LD);
    if (b.Tmp <= b.Tep || b.H_liquidus <= b.Tep || (C == 0.0 && b.H_liquidus <= b.Tmp))
        throw Fail{ORC_OVERFLOW};
    return b;
}

// eutectic_rescaled.cpp:95-105; region numbering as eutectic_rescaled.h:43-50.
int region_of(double H, double C, const orc_bounds& b) {
    if (C == 0.0) {
        if (H <= b.Tmp) return 1;          // PureSolid
        if (H < b.H_liquidus) return 6;    // PureMelting
        return 5;                          // Liquid
    }
    if (H <= b.Tep) return 2;              // TwoSolids
    if (H >= b.H_liquidus) return 5;       // Liquid
    if (H <= b.H_eutectic_end) return 3;   // Eutectic
    return 4;                              // SolidLiquid
}

// eutectic_rescaled.cpp:108-114
double clip_fraction(lc v) {
    const lc tol = 64.0L * std::numeric_limits<double>::epsilon();
    if (!std::isfinite(v) || v < -tol || v > 1.0L + tol) throw Fail{ORC_RUNTIME};
    return (double)std::min(std::max(v, (lc)0), (lc)1);
}

// eutectic_rescaled.cpp:116-121
double minus_magnitude(lc m) {
    if (m > (lc)std::numeric_limits<double>::max()) return -std::numeric_limits<double>::infinity();
    return -(double)m;
}

orc_phase evaluate_or_throw(const orc_material& p, const orc_derived& d, double H, double C, double P) {
    finite_or_throw(H);
    const orc_bounds b = bounds_or_throw(p, d, C, P);
    const lc LD = d.LD;
    const lc Xe = p.Xe;
    orc_phase s{};
    s.region = region_of(H, C, b);
    s.Tep = b.Tep;
    switch (s.region) {
    case 1:
        s.phi1 = 1.0; s.TDp = H; s.dTD_dHD = 1.0;
        break;
    case 6:
        s.phil = clip_fraction(((lc)H - b.Tmp) / LD);
        s.phi1 = 1.0 - s.phil;
        s.TDp = b.Tmp;
        break;
    case 2:
        s.phi1 = 1.0 - C; s.phi2 = C; s.TDp = H; s.dTD_dHD = 1.0;
        break;
    case 3: {
        const lc cap = (lc)C / Xe;
        const lc melt = (H == b.H_eutectic_end) ? cap : std::min(cap, ((lc)H - b.Tep) / LD);
        const lc second = std::max((lc)0, (lc)C - melt * Xe);
        s.phil = clip_fraction(melt);
        s.phi2 = clip_fraction(second);
        s.phi1 = clip_fraction(1.0L - melt - second);
        s.cl = p.Xe;
        s.TDp = b.Tep;
        break;
    }
    case 4: {
        // LD*phi^2 - (H - Tmp)*phi - C/Xe = 0, cancellation-free root choice.
        const lc a = (lc)H - b.Tmp;
        const lc r = (lc)C / Xe;
        const lc disc = std::hypot(a, 2.0L * std::sqrt(LD) * std::sqrt(r));
        const lc melt = a >= 0.0L ? (a + disc) / (2.0L * LD) : 2.0L * r / (disc - a);
        s.phil = clip_fraction(melt);
        s.phi1 = clip_fraction(1.0L - melt);
        s.cl = clip_fraction((lc)C / melt);
        s.TDp = to_double_checked(a >= 0.0L ? (lc)b.Tmp - r / melt : (lc)H - LD * melt);
        s.dTD_dHD = clip_fraction(a >= 0.0L ? 2.0L * (LD / disc) * (r / (disc + a))
                                            : 0.5L * (1.0L - a / disc));
        s.dTD_dCD = minus_magnitude((LD / disc) / Xe);
        break;
    }
    case 5:
        s.phil = 1.0; s.cl = C;
        s.TDp = to_double_checked((lc)H - LD);
        s.dTD_dHD = 1.0;
        break;
    }
    if (C == 0.0 && H > b.Tep && s.region != 5) {
        const lc gap = std::fabs((lc)H - b.Tmp);
        s.dTD_dCD = gap == 0.0L ? -std::numeric_limits<double>::infinity()
                                : minus_magnitude((LD / gap) / Xe);
    }
    const double solid = s.phi1 + s.phi2;
    s.has_solid = solid > 0.0;
    s.has_liquid = s.phil > 0.0;
    s.cs = s.has_solid ? s.phi2 / solid : 0.0;
    if (!s.has_liquid) s.cl = 0.0;
    s.finite_temperature_derivatives = std::isfinite(s.dTD_dCD) && std::isfinite(s.dTD_dHD);
    return s;
}

}  // namespace

extern "C" int orc_phase_derive(const orc_material* m, orc_derived* d) {
    try { *d = derive_or_throw(*m); return ORC_OK; } catch (const Fail& f) { return f.code; }
}

extern "C" int orc_phase_boundaries(const orc_material* m, double C, double P, orc_bounds* b) {
    try {
        const orc_derived d = derive_or_throw(*m);
        *b = bounds_or_throw(*m, d, C, P);
        return ORC_OK;
    } catch (const Fail& f) { return f.code; }
}

extern "C" int orc_phase_evaluate(const orc_material* m, double H, double C, double P, orc_phase* s) {
    try {
        const orc_derived d = derive_or_throw(*m);
        *s = evaluate_or_throw(*m, d, H, C, P);
        return ORC_OK;
    } catch (const Fail& f) { return f.code; }
}

extern "C" int orc_phase_classify(const orc_material* m, double H, double C, double P, int* region) {
    try {
        const orc_derived d = derive_or_throw(*m);
        finite_or_throw(H);
        *region = region_of(H, C, bounds_or_throw(*m, d, C, P));
        return ORC_OK;
    } catch (const Fail& f) { return f.code; }
}

extern "C" int orc_phase_evaluate_batch(const orc_material* m, const double* H, const double* C,
                                        const double* P, double P_const, size_t n,
                                        orc_phase* out, long long* first_bad) {
    orc_derived d;
    try { d = derive_or_throw(*m); } catch (const Fail& f) { if (first_bad) *first_bad = -1; return f.code; }
    int code = ORC_OK;
    long long bad = -1;
    const double nan = std::numeric_limits<double>::quiet_NaN();
    for (size_t i = 0; i < n; ++i) {
        try {
            out[i] = evaluate_or_throw(*m, d, H[i], C[i], P ? P[i] : P_const);
        } catch (const Fail& f) {
            orc_phase z{};
            z.phi1 = z.phi2 = z.phil = z.cl = z.cs = z.TDp = z.Tep = z.dTD_dCD = z.dTD_dHD = nan;
            out[i] = z;
            if (bad < 0) { bad = (long long)i; code = f.code; }
        }
    }
    if (first_bad) *first_bad = bad;
    return code;
}

// Exported for the transport restatement in this library.
namespace orc_internal {
bool phase_eval(const orc_material& m, const orc_derived& d, double H, double C, double P,
                orc_phase& s, int& code) {
    try { s = evaluate_or_throw(m, d, H, C, P); return true; }
    catch (const Fail& f) { code = f.code; return false; }
}
bool derive(const orc_material& m, orc_derived& d) {
    try { d = derive_or_throw(m); return true; } catch (const Fail&) { return false; }
}
}  // namespace orc_internal
