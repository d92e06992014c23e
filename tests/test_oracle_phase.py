"""The phase oracle against the reference: bitwise pins and known answers."""
import dataclasses
import math

import numpy as np
import pytest

import phase_known_answers as ka
from oracle import pyoracle as po

GOLDEN = np.load(__import__("os").path.join(__import__("os").path.dirname(__file__), "golden", "phase_golden.npz"))
FIELDS = ["phi1", "phi2", "phil", "cl", "cs", "TDp", "Tep", "dTD_dCD", "dTD_dHD"]


class OracleModel:
    """EutecticModel-shaped view of an oracle library."""

    def __init__(self, p, lib=None):
        self.p = p
        self.o = po.PhaseOracle(p, lib)

    def derived(self):
        return self.o.derived()

    def boundaries(self, C, P):
        code, b = self.o.boundaries(C, P)
        assert code == 0
        return type("B", (), b)

    def evaluate(self, H, C, P):
        code, s = self.o.evaluate(H, C, P)
        if code:
            raise ValueError(code)
        return type("S", (), s)

    def classify(self, H, C, P):
        code, r = self.o.classify(H, C, P)
        assert code == 0
        return r


def _batch(lib, set_index):
    p = ka.parameter_sets()[set_index]
    sel = GOLDEN["set"] == set_index
    o = po.PhaseOracle(p, lib)
    code, bad, out = o.evaluate_batch(GOLDEN["H"][sel], GOLDEN["C"][sel], GOLDEN["P"][sel])
    return sel, out


@pytest.mark.parametrize("set_index", [0, 1, 2])
def test_restated_phase_equals_golden_bitwise(set_index):
    """Every golden state: same status, same region and bit-identical fields."""
    sel, out = _batch(po.restated(), set_index)
    status = GOLDEN["status"][sel]
    ok = status == 0
    for f in FIELDS:
        a, b = out[f][ok], GOLDEN[f][sel][ok]
        assert np.array_equal(a.view(np.int64), b.view(np.int64)), f
    assert np.array_equal(out["region"][ok], GOLDEN["region"][sel][ok])
    # invalid inputs are rejected as std::invalid_argument (class 1)
    assert np.all(np.isnan(out["TDp"][~ok]))


def test_restated_error_classes():
    p = ka.parameter_sets()[0]
    o = po.PhaseOracle(p)
    assert o.evaluate(1.0, p.Xe * 1.5, 0.0)[0] == 1
    assert o.evaluate(1.0, -1e-3, 0.0)[0] == 1
    assert o.evaluate(float("nan"), 0.1, 0.0)[0] == 1
    bad = dataclasses.replace(p, Xe=1.5)
    assert po.PhaseOracle(bad).evaluate(1.0, 0.1, 0.0)[0] == 1
    # huge pressure: pressure-corrected temperature overflows
    assert o.evaluate(1.0, 0.1, 1e308)[0] == 2


@pytest.mark.skipif(not po.reference_available(), reason="reference build (oracle/_ref) not present")
def test_restated_phase_equals_reference_random():
    rng = np.random.default_rng(5)
    for p in ka.parameter_sets():
        for P in ka.PRESSURES:
            n = 3000
            H = rng.uniform(-1, 6, n)
            C = np.where(rng.random(n) < 0.5, rng.uniform(0, p.Xe, n), p.Xe * 10.0 ** (-300 * rng.random(n)))
            C[:50] = 0.0
            a = po.PhaseOracle(p, po.restated()).evaluate_batch(H, C, None, P)
            b = po.PhaseOracle(p, po.reference()).evaluate_batch(H, C, None, P)
            assert a[0] == b[0] and a[1] == b[1]
            for f in FIELDS:
                assert np.array_equal(a[2][f].view(np.int64), b[2][f].view(np.int64)), f


@pytest.mark.parametrize("set_index", [0, 1, 2])
def test_oracle_known_answers(set_index):
    p = ka.parameter_sets()[set_index]
    m = OracleModel(p)
    for P in ka.PRESSURES:
        for H, C, exp in ka.region_cases(m, p, P):
            s = m.evaluate(H, C, P)
            ka.check_state(m, s, H, C, P, p)
            assert s.region == exp["region"] == m.classify(H, C, P)
            for k, v in exp.items():
                if k != "region":
                    ka.near(getattr(s, k), v, k)


@pytest.mark.parametrize("set_index", [0, 1, 2])
def test_oracle_interface_continuity_and_ownership(set_index):
    p = ka.parameter_sets()[set_index]
    m = OracleModel(p)
    for P in ka.PRESSURES:
        for C, lo, at, hi in ka.boundary_points(m, p, P):
            sl, sa, sh = m.evaluate(lo, C, P), m.evaluate(at, C, P), m.evaluate(hi, C, P)
            for s, H in ((sl, lo), (sa, at), (sh, hi)):
                ka.check_state(m, s, H, C, P, p)
            ka.near(sl.TDp, sa.TDp, "T continuity below")
            ka.near(sh.TDp, sa.TDp, "T continuity above")
            ka.near(sl.phil, sa.phil, "phi continuity below")
            ka.near(sh.phil, sa.phil, "phi continuity above")
            assert m.classify(m.boundaries(C, P).H_liquidus, C, P) == 5
        C = 0.4 * p.Xe
        b = m.boundaries(C, P)
        assert m.classify(b.Tep, C, P) == 2
        assert m.classify(np.nextafter(b.Tep, np.inf), C, P) == 3
        assert m.classify(b.H_eutectic_end, C, P) == 3
        assert m.classify(np.nextafter(b.H_eutectic_end, np.inf), C, P) == 4
        assert m.classify(np.nextafter(b.H_liquidus, -np.inf), C, P) == 4
        pure = m.boundaries(0.0, P)
        corner = m.evaluate(pure.Tmp, 0.0, P)
        assert corner.region == 1 and not corner.finite_temperature_derivatives and corner.dTD_dCD == -math.inf


def test_oracle_pinned_scales():
    m = OracleModel(ka.parameter_sets()[0])
    d = m.derived()
    ka.near(d["dT"], 520.0, "dT")
    ka.near(d["h0"], 624000.0, "h0")
    ka.near(d["TDm0"], 50.0 / 13.0, "TDm0")
    ka.near(d["TDe0"], 37.0 / 13.0, "TDe0")
    ka.near(d["LD"], 125.0 / 156.0, "LD")


def test_oracle_derivatives_finite_difference():
    """dT/dH and dT/dC against centred differences (test_eutectic.cpp:256-280)."""
    for p in ka.parameter_sets():
        m = OracleModel(p)
        for P in ka.PRESSURES:
            C = 0.4 * p.Xe
            b = m.boundaries(C, P)
            for H in (b.Tep - 0.2, (b.Tep + b.H_eutectic_end) / 2, (b.H_eutectic_end + b.H_liquidus) / 2, b.H_liquidus + 0.2):
                s = m.evaluate(H, C, P)
                h = 1e-6
                fdH = (m.evaluate(H + h, C, P).TDp - m.evaluate(H - h, C, P).TDp) / (2 * h)
                fdC = (m.evaluate(H, C + h, P).TDp - m.evaluate(H, C - h, P).TDp) / (2 * h)
                ka.near(s.dTD_dHD, fdH, "dT/dH", 2e-8, 2e-8)
                ka.near(s.dTD_dCD, fdC, "dT/dC", 2e-8, 2e-8)
