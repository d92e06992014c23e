"""Known-answer phase cases restated from the reference's own phase test.

src/phase/test/test_eutectic.cpp builds its answers by forward construction
(choose T and the liquid fraction, then form H and C) and checks the
inversion against them (:122-183), checks interface ownership and
continuity with nextafter neighbours (:185-235), conservation invariants of
every state (:89-120), derivatives by finite differences (:256-308) and the
pinned scales (:326-332). This module regenerates those cases for any
evaluator with the EutecticModel interface (evaluate, classify, boundaries,
derived); the tolerances are the reference test's (rtol 3e-12, atol 3e-13).
"""
from __future__ import annotations

import math

import numpy as np

from mantlepar_b200.synthetic import Material

PRESSURES = (0.0, 1.0e5, 1.0e9, -1.0e7)
RTOL, ATOL = 3.0e-12, 3.0e-13


def alternative() -> Material:
    return Material(Tm0=2100.0, Te0=1500.0, cp=1350.0, L=6.0e5, Xe=0.3, nu=8.0e6, rho=3100.0,
                    rhor=450.0, mus=3.0e19, mul=2.0, k0=2.0e-8, g=9.81, alpha0=4.0e-5)


def parameter_sets() -> list[Material]:
    alt = alternative()
    neg = alternative()
    neg.nu = -neg.nu
    return [Material(), alt, neg]


def near(actual, expected, name, rtol=RTOL, atol=ATOL):
    tol = atol + rtol * max(abs(actual), abs(expected))
    assert math.isfinite(actual) and math.isfinite(expected) and abs(actual - expected) <= tol, \
        f"{name}: got {actual!r}, expected {expected!r}, tolerance {tol}"


def check_state(model, s, H, C, P, p: Material):
    """Invariants every state must satisfy (test_eutectic.cpp:89-120)."""
    d = model.derived()
    for v in (s.phi1, s.phi2, s.phil, s.cs, s.cl):
        assert math.isfinite(v) and 0.0 <= v <= 1.0, f"fraction out of range at H={H} C={C} P={P}"
    near(s.phi1 + s.phi2 + s.phil, 1.0, "Total phase fraction")
    near(s.TDp + d["LD"] * s.phil, H, "Enthalpy conservation")
    near(s.phi2 + s.phil * s.cl, C, "Composition conservation", RTOL, 0.0)
    assert s.has_solid == (s.phi1 + s.phi2 > 0.0)
    assert s.has_liquid == (s.phil > 0.0)
    if s.has_solid:
        near(s.cs * (s.phi1 + s.phi2), s.phi2, "Solid composition balance")
    else:
        assert s.cs == 0.0
    if not s.has_liquid:
        assert s.cl == 0.0
    near(s.Tep, (p.Te0 + P / p.nu) / d["dT"], "Pressure-corrected eutectic temperature")
    assert math.isfinite(s.dTD_dHD) and 0.0 <= s.dTD_dHD <= 1.0
    assert not math.isnan(s.dTD_dCD) and s.dTD_dCD <= 0.0
    assert s.finite_temperature_derivatives == math.isfinite(s.dTD_dCD)


def region_cases(model, p: Material, P: float):
    """(H, C, expected) triples of test_eutectic.cpp:122-183 (regions())."""
    d = model.derived()
    LD = d["LD"]
    C = 0.4 * p.Xe
    b = model.boundaries(C, P)
    out = [(b.Tep - 0.25, C, dict(region=2, phi1=1.0 - C, phi2=C, phil=0.0))]
    for liquid in (0.1, 0.2, 0.3):
        out.append((b.Tep + LD * liquid, C, dict(region=3, TDp=b.Tep, phil=liquid, phi2=C - liquid * p.Xe, cl=p.Xe)))
    for offset in (0.15, 0.5, 0.85):
        for liquid in (0.05, 0.3, 0.8, 0.99):
            T = b.Tep + offset
            cl = p.Xe * (1.0 - offset)
            out.append((T + LD * liquid, liquid * cl, dict(region=4, TDp=T, phil=liquid, cl=cl, phi2=0.0)))
    out.append((b.H_liquidus + 0.3, C, dict(region=5, phil=1.0, cl=C)))
    pure = model.boundaries(0.0, P)
    out.append((pure.Tmp - 0.3, 0.0, dict(region=1, phi1=1.0)))
    for liquid in (0.1, 0.5, 0.9):
        out.append((pure.Tmp + LD * liquid, 0.0, dict(region=6, phil=liquid, TDp=pure.Tmp)))
    out.append((pure.H_liquidus + 0.2, 0.0, dict(region=5)))
    eut = model.boundaries(p.Xe, P)
    out.append((eut.Tep + 0.5 * LD, p.Xe, dict(region=3, phil=0.5)))
    return out


def boundary_points(model, p: Material, P: float):
    """nextafter triples at every interval end (test_eutectic.cpp:189-201)."""
    pts = []
    for C in (0.0, 1.0e-300, 1.0e-18, 0.4 * p.Xe, float(np.nextafter(p.Xe, 0.0)), p.Xe):
        b = model.boundaries(C, P)
        for H in (b.Tep, b.Tmp, b.H_eutectic_end, b.H_liquidus):
            pts.append((C, float(np.nextafter(H, -np.inf)), H, float(np.nextafter(H, np.inf))))
    return pts


def conservation_states(p: Material, P: float, model, count: int, seed: int):
    """Seeded random states shaped like test_eutectic.cpp:237-254: C alternates
    ordinary mixtures and trace amounts down to ~1e-301; H spans the solidus to
    beyond the liquidus."""
    rng = np.random.default_rng(seed)
    d = model.derived()
    b = model.boundaries(0.4 * p.Xe, P)
    u = rng.random((count, 2))
    C = np.where(np.arange(count) % 2 == 0, p.Xe * u[:, 0], p.Xe * 10.0 ** (-300.0 * u[:, 0]))
    H = b.Tep - 0.5 + (2.0 + d["LD"]) * u[:, 1]
    return H, C
