// Binary eutectic equilibrium in FP64 for B200 kernels (and host setup).
//
// Same closed forms and branch ownership as the reference's
// EutecticModel::evaluate (src/phase/eutectic_rescaled.cpp:192-282,
// boundaries :163-185, selectRegion :95-105, unitFraction :108-114), written
// for a GPU: no long double (the reference's 80-bit intermediates become
// FP64), no exceptions (a status code per point), reciprocals hoisted where
// one division serves several quotients. The interval ends (boundaries) use
// explicitly rounded operations so the host's mp_phase_boundaries() and the
// kernels select regions from bit-identical values.
#ifndef MP_PHASE_MATH_CUH
#define MP_PHASE_MATH_CUH

#include <math.h>
#include <stdint.h>

#ifdef __CUDACC__
#define MP_HD __host__ __device__ __forceinline__
#else
#define MP_HD inline
#endif

#if defined(__CUDA_ARCH__)
#define MP_ADD(a, b) __dadd_rn((a), (b))
#define MP_SUB(a, b) __dsub_rn((a), (b))
#define MP_MUL(a, b) __dmul_rn((a), (b))
#define MP_DIV(a, b) __ddiv_rn((a), (b))
#else
#define MP_ADD(a, b) ((a) + (b))
#define MP_SUB(a, b) ((a) - (b))
#define MP_MUL(a, b) ((a) * (b))
#define MP_DIV(a, b) ((a) / (b))
#endif

namespace mp {

// Per-point status codes (0 ok); values match mp_status.
enum : int { PH_OK = 0, PH_INVALID = 101, PH_OVERFLOW = 102, PH_RUNTIME = 103 };

enum : int { R_PURE_SOLID = 1, R_TWO_SOLIDS = 2, R_EUTECTIC = 3, R_SOLID_LIQUID = 4, R_LIQUID = 5, R_PURE_MELTING = 6 };

// Model constants the kernels need (derived once on the host).
struct PhaseConst {
    double Xe, LD, sqrtLD, TDe0, nu, dT;
};

struct Bounds {
    double Tep, Tmp, Heut, Hliq;
};

struct PhaseOut {
    double phi1, phi2, phil, cl, cs, T, Tep, dTdC, dTdH;
    int region;
    int flags;  // bit0 has_solid, bit1 has_liquid, bit2 finite derivatives
};

MP_HD bool mp_isfinite(double x) { return isfinite(x); }

MP_HD double max_double() { return 1.7976931348623157e308; }

// Pressure-corrected eutectic temperature TDe0 + P/nu/dT (eutectic_rescaled.cpp:143-149).
MP_HD int eutectic_temperature(const PhaseConst& k, double P, double& Tep) {
    if (!mp_isfinite(P)) return PH_INVALID;
    const double shift = MP_DIV(MP_DIV(P, k.nu), k.dT);
    Tep = MP_ADD(k.TDe0, shift);
    if (!mp_isfinite(Tep)) return PH_OVERFLOW;
    return PH_OK;
}

// Interval ends for composition C at eutectic temperature Tep (eutectic_rescaled.cpp:163-185).
MP_HD int bounds_at(const PhaseConst& k, double C, double Tep, Bounds& b) {
    if (!mp_isfinite(C) || C < 0.0 || C > k.Xe) return PH_INVALID;
    b.Tep = Tep;
    b.Tmp = MP_ADD(Tep, 1.0);
    const double r = MP_DIV(C, k.Xe);
    b.Heut = MP_ADD(Tep, MP_MUL(k.LD, r));
    b.Hliq = MP_ADD(MP_ADD(Tep, MP_SUB(1.0, r)), k.LD);
    if (C == 0.0) b.Hliq = MP_ADD(b.Tmp, k.LD);
    if (!mp_isfinite(b.Tmp) || !mp_isfinite(b.Heut) || !mp_isfinite(b.Hliq)) return PH_OVERFLOW;
    if (b.Tmp <= b.Tep || b.Hliq <= b.Tep || (C == 0.0 && b.Hliq <= b.Tmp)) return PH_OVERFLOW;
    return PH_OK;
}

// Region ownership at the interfaces (eutectic_rescaled.cpp:95-105).
MP_HD int region_of(double H, double C, const Bounds& b) {
    if (C == 0.0) {
        if (H <= b.Tmp) return R_PURE_SOLID;
        if (H < b.Hliq) return R_PURE_MELTING;
        return R_LIQUID;
    }
    if (H <= b.Tep) return R_TWO_SOLIDS;
    if (H >= b.Hliq) return R_LIQUID;
    if (H <= b.Heut) return R_EUTECTIC;
    return R_SOLID_LIQUID;
}

// Clip roundoff excursions of a fraction; larger ones are errors (eutectic_rescaled.cpp:108-114).
MP_HD double clip_fraction(double v, int& st) {
    const double tol = 64.0 * 2.220446049250313e-16;
    if (!(v >= -tol && v <= 1.0 + tol)) { st = PH_RUNTIME; return v; }
    return v < 0.0 ? 0.0 : (v > 1.0 ? 1.0 : v);
}

MP_HD double minus_magnitude(double m) { return m > max_double() ? -INFINITY : -m; }

// Full evaluation. Returns a status; outputs are meaningful only when 0.
MP_HD int phase_eval(const PhaseConst& k, double H, double C, double Tep, PhaseOut& s) {
    if (!mp_isfinite(H)) return PH_INVALID;
    Bounds b;
    int st = bounds_at(k, C, Tep, b);
    if (st) return st;
    const double LD = k.LD, Xe = k.Xe;
    s.phi1 = s.phi2 = s.phil = s.cl = s.cs = 0.0;
    s.dTdC = s.dTdH = 0.0;
    s.Tep = b.Tep;
    s.region = region_of(H, C, b);
    switch (s.region) {
    case R_PURE_SOLID:
        s.phi1 = 1.0; s.T = H; s.dTdH = 1.0;
        break;
    case R_PURE_MELTING:
        s.phil = clip_fraction((H - b.Tmp) / LD, st);
        s.phi1 = 1.0 - s.phil;
        s.T = b.Tmp;
        break;
    case R_TWO_SOLIDS:
        s.phi1 = 1.0 - C; s.phi2 = C; s.T = H; s.dTdH = 1.0;
        break;
    case R_EUTECTIC: {
        const double cap = C / Xe;
        const double melt = (H == b.Heut) ? cap : fmin(cap, (H - b.Tep) / LD);
        const double second = fmax(0.0, C - melt * Xe);
        s.phil = clip_fraction(melt, st);
        s.phi2 = clip_fraction(second, st);
        s.phi1 = clip_fraction(1.0 - melt - second, st);
        s.cl = Xe;
        s.T = b.Tep;
        break;
    }
    case R_SOLID_LIQUID: {
        // LD*phi^2 - (H - Tmp)*phi - C/Xe = 0 with the cancellation-free root.
        const double a = H - b.Tmp;
        const double r = C / Xe;
        const double disc = hypot(a, 2.0 * k.sqrtLD * sqrt(r));
        const double melt = a >= 0.0 ? (a + disc) / (2.0 * LD) : 2.0 * r / (disc - a);
        const double inv = 1.0 / melt;
        s.phil = clip_fraction(melt, st);
        s.phi1 = clip_fraction(1.0 - melt, st);
        s.cl = clip_fraction(C * inv, st);
        s.T = a >= 0.0 ? b.Tmp - r * inv : H - LD * melt;
        const double q = LD / disc;
        s.dTdH = clip_fraction(a >= 0.0 ? 2.0 * q * (r / (disc + a)) : 0.5 * (1.0 - a / disc), st);
        s.dTdC = minus_magnitude(q / Xe);
        break;
    }
    case R_LIQUID:
        s.phil = 1.0; s.cl = C; s.T = H - LD; s.dTdH = 1.0;
        break;
    }
    if (!mp_isfinite(s.T)) st = st ? st : PH_OVERFLOW;
    if (C == 0.0 && H > b.Tep && s.region != R_LIQUID) {
        const double gap = fabs(H - b.Tmp);
        s.dTdC = gap == 0.0 ? -INFINITY : minus_magnitude((LD / gap) / Xe);
    }
    const double solid = s.phi1 + s.phi2;
    const bool has_solid = solid > 0.0, has_liquid = s.phil > 0.0;
    s.cs = has_solid ? s.phi2 / solid : 0.0;
    if (!has_liquid) s.cl = 0.0;
    const bool fin = mp_isfinite(s.dTdC) && mp_isfinite(s.dTdH);
    s.flags = (has_solid ? 1 : 0) | (has_liquid ? 2 : 0) | (fin ? 4 : 0);
    return st;
}

// Lean form for the transport stage: T, phil, cl, cs, dT/dC only (same
// arithmetic as phase_eval for those outputs).
struct PhaseLean {
    double T, phil, cl, cs, dTdC;
};

MP_HD int phase_lean(const PhaseConst& k, double H, double C, const Bounds& b, PhaseLean& s) {
    int st = PH_OK;
    const double LD = k.LD, Xe = k.Xe;
    double phi1 = 0.0, phi2 = 0.0;
    s.phil = 0.0; s.cl = 0.0; s.dTdC = 0.0;
    const int region = region_of(H, C, b);
    switch (region) {
    case R_PURE_SOLID:
        phi1 = 1.0; s.T = H;
        break;
    case R_PURE_MELTING:
        s.phil = clip_fraction((H - b.Tmp) / LD, st);
        phi1 = 1.0 - s.phil;
        s.T = b.Tmp;
        break;
    case R_TWO_SOLIDS:
        phi1 = 1.0 - C; phi2 = C; s.T = H;
        break;
    case R_EUTECTIC: {
        const double cap = C / Xe;
        const double melt = (H == b.Heut) ? cap : fmin(cap, (H - b.Tep) / LD);
        const double second = fmax(0.0, C - melt * Xe);
        s.phil = clip_fraction(melt, st);
        phi2 = clip_fraction(second, st);
        phi1 = clip_fraction(1.0 - melt - second, st);
        s.cl = Xe;
        s.T = b.Tep;
        break;
    }
    case R_SOLID_LIQUID: {
        const double a = H - b.Tmp;
        const double r = C / Xe;
        const double disc = hypot(a, 2.0 * k.sqrtLD * sqrt(r));
        const double melt = a >= 0.0 ? (a + disc) / (2.0 * LD) : 2.0 * r / (disc - a);
        const double inv = 1.0 / melt;
        s.phil = clip_fraction(melt, st);
        phi1 = clip_fraction(1.0 - melt, st);
        s.cl = clip_fraction(C * inv, st);
        s.T = a >= 0.0 ? b.Tmp - r * inv : H - LD * melt;
        s.dTdC = minus_magnitude((LD / disc) / Xe);
        break;
    }
    case R_LIQUID:
        s.phil = 1.0; s.cl = C; s.T = H - LD;
        break;
    }
    if (C == 0.0 && H > b.Tep && region != R_LIQUID) {
        const double gap = fabs(H - b.Tmp);
        s.dTdC = gap == 0.0 ? -INFINITY : minus_magnitude((LD / gap) / Xe);
    }
    const double solid = phi1 + phi2;
    s.cs = solid > 0.0 ? phi2 / solid : 0.0;
    if (!(s.phil > 0.0)) s.cl = 0.0;
    return st;
}

// Constants of the stage kernels' phase evaluation (precomputed reciprocals).
struct StageConst {
    double Xe, LD, invXe, invLD, halfInvLD, fourLD, LDoverXe;
};

MP_HD StageConst stage_const(const PhaseConst& k) {
    StageConst c;
    c.Xe = k.Xe; c.LD = k.LD;
    c.invXe = 1.0 / k.Xe; c.invLD = 1.0 / k.LD; c.halfInvLD = 0.5 / k.LD;
    c.fourLD = 4.0 * k.LD; c.LDoverXe = k.LD / k.Xe;
    return c;
}

// Phase evaluation for the transport stage: the same regions and closed
// forms as phase_eval, with the divisions by Xe and LD replaced by
// precomputed reciprocals. kFull = false evaluates T and phil only (the cell
// quadrature), still applying every admissibility check of the full
// evaluation; kFull = true adds cl, cs and dT/dC (the face points).
//  - solid + liquid: T = Tmp - (disc - a)/2 is the reference's
//    Tmp - r/melt (a >= 0) and H - LD*melt (a < 0) on the quadratic
//    melt^2 LD - a melt - r = 0; its rounding error is bounded by that of
//    disc, far below T >= Tep. 1/g (g = disc - a) and 1/(r disc) come from
//    one division where that product is in range.
//  - two solids: (1 - C) + C rounds to exactly 1 for 0 <= C <= 1, so
//    cs = phi2/solid = C.
// Agrees with phase_eval to a few ulp; region selection uses interval ends
// formed the same way.
template <bool kFull>
MP_HD int phase_stage_t(const StageConst& k, double H, double C, double Tep, PhaseLean& s) {
    if (!(C >= 0.0 && C <= k.Xe) || !mp_isfinite(H)) return PH_INVALID;
    int st = PH_OK;
    const double Tmp = Tep + 1.0;
    const double r = C * k.invXe;
    const double Hliq = C == 0.0 ? Tmp + k.LD : (Tep + (1.0 - r)) + k.LD;
    const double Heut = Tep + k.LD * r;
    double phi1 = 0.0, phi2 = 0.0;
    s.phil = 0.0; s.cl = 0.0; s.cs = 0.0; s.dTdC = 0.0;
    bool liquid_region = false, general_cs = false;
    if (C == 0.0) {
        if (H <= Tmp) { phi1 = 1.0; s.T = H; }
        else if (H < Hliq) {
            s.phil = clip_fraction((H - Tmp) * k.invLD, st);
            phi1 = 1.0 - s.phil;
            s.T = Tmp;
        } else { s.phil = 1.0; s.T = H - k.LD; liquid_region = true; }
    } else if (H <= Tep) {
        phi1 = 1.0 - C; phi2 = C; s.T = H;
        if (kFull) {
            if (phi1 + phi2 == 1.0) s.cs = C;
            else general_cs = true;
        }
    } else if (H >= Hliq) {
        s.phil = 1.0; s.cl = C; s.T = H - k.LD; liquid_region = true;
    } else if (H <= Heut) {
        const double melt = (H == Heut) ? r : fmin(r, (H - Tep) * k.invLD);
        const double second = fmax(0.0, C - melt * k.Xe);
        s.phil = clip_fraction(melt, st);
        phi2 = clip_fraction(second, st);
        phi1 = clip_fraction(1.0 - melt - second, st);
        s.cl = k.Xe;
        s.T = Tep;
        general_cs = kFull;
    } else {
        const double a = H - Tmp;
        const double disc = fabs(a) < 1e150 ? sqrt(a * a + k.fourLD * r) : hypot(a, 2.0 * sqrt(k.LD * r));
        double melt;
        if (kFull) {
            double inv_melt, inv_disc;
            if (a >= 0.0) {
                melt = (a + disc) * k.halfInvLD;
                const double inv = 1.0 / (melt * disc);
                inv_melt = disc * inv; inv_disc = melt * inv;
            } else {
                const double g = disc - a, rd = r * disc, p = g * rd;
                if (p > 1e-290 && p < 1e290) {
                    const double x = 1.0 / p;
                    const double inv_rd = g * x;
                    melt = 2.0 * r * (rd * x);
                    inv_melt = 0.5 * g * (disc * inv_rd);
                    inv_disc = r * inv_rd;
                } else {
                    melt = 2.0 * r / g;
                    const double inv = 1.0 / (melt * disc);
                    inv_melt = disc * inv; inv_disc = melt * inv;
                }
            }
            s.cl = clip_fraction(C * inv_melt, st);
            s.dTdC = minus_magnitude(k.LDoverXe * inv_disc);
        } else {
            melt = a >= 0.0 ? (a + disc) * k.halfInvLD : 2.0 * r / (disc - a);
            // cl = C/melt in [-tol, 1 + tol] (C, melt > 0), as the full evaluation checks.
            if (!(C <= (1.0 + 64.0 * 2.220446049250313e-16) * melt)) st = PH_RUNTIME;
        }
        s.phil = clip_fraction(melt, st);
        phi1 = clip_fraction(1.0 - melt, st);
        s.T = Tmp - 0.5 * (disc - a);
    }
    if (kFull) {
        if (C == 0.0 && H > Tep && !liquid_region) {
            const double gap = fabs(H - Tmp);
            s.dTdC = gap == 0.0 ? -INFINITY : minus_magnitude(k.LDoverXe / gap);
        }
        if (general_cs) {
            const double solid = phi1 + phi2;
            s.cs = (solid > 0.0 && phi2 != 0.0) ? phi2 / solid : 0.0;
        }
        if (!(s.phil > 0.0)) s.cl = 0.0;
    }
    return st;
}

MP_HD int phase_stage(const StageConst& k, double H, double C, double Tep, PhaseLean& s) {
    return phase_stage_t<true>(k, H, C, Tep, s);
}
MP_HD int phase_stage_lean(const StageConst& k, double H, double C, double Tep, PhaseLean& s) {
    return phase_stage_t<false>(k, H, C, Tep, s);
}

}  // namespace mp

#endif
