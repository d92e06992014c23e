"""Transport on general quad meshes: the restated oracle against the
reference-backed golden runs, and the mesh families' vertices."""
import os

import numpy as np
import pytest

from oracle import pyoracle as po
from mantlepar_b200 import synthetic as sy
import quad_cases as qc

GOLDEN = np.load(os.path.join(os.path.dirname(__file__), "golden", "quads_golden.npz"))


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float64).view(np.int64)


@pytest.mark.parametrize("name", qc.QUAD_CASES)
def test_restated_quads_equal_golden_bitwise(name):
    t, xy, _, _ = qc.quad_oracle(name)
    assert np.array_equal(bits(xy), bits(GOLDEN[f"{name}_xy"]))
    code, r = t.rhs()
    assert code == 0
    for k in ["rhsH", "rhsC", "T", "phi", "rate"]:
        assert np.array_equal(bits(r[k]), bits(GOLDEN[f"{name}_rhs_{k}"])), k
    code, a, b = t.limiter()
    assert code == 0
    assert np.array_equal(bits(a), bits(GOLDEN[f"{name}_thetaH"])) and np.array_equal(bits(b), bits(GOLDEN[f"{name}_thetaC"]))
    t, _, _, _ = qc.quad_oracle(name)
    code, reps = t.step(10)
    assert code == 0
    assert np.array_equal(bits(np.stack(t.get_state())), bits(GOLDEN[f"{name}_rk3_10"]))
    assert np.array_equal(bits([x["dt"] for x in reps]), bits(GOLDEN[f"{name}_rk3_10_dt"]))


def test_quad_meshes_differ_from_uniform():
    """The perturbed mesh is not the uniform one: cell averages are advanced
    differently, and the limiter acts on different points."""
    t, _, _, _ = qc.quad_oracle("p12x10")
    _, r = t.rhs()
    w = qc.quad_case("p12x10")[0]
    u = po.TransportOracle(sy.material_s(), w, integrator=3)
    u.set_face_velocity(*sy.face_velocity(w))
    u.set_state(*sy.initial_state(w))
    _, ru = u.rhs()
    assert np.max(np.abs(r["rhsH"] - ru["rhsH"])) > 1e-3


@pytest.mark.parametrize("family,pert", [(1, 0.2), (1, 0.0), (2, 0.0), (0, 0.0)])
def test_mesh_vertices_of_every_generator_agree(family, pert):
    """VertexAt (src/core/mesh.cpp:27-55) three ways: the library's host
    function, the numpy builder and the oracle's mesh; bit for bit."""
    from mantlepar_b200.transport import mesh_vertices
    w = sy.Workload(nx=9, ny=7)
    a = mesh_vertices(w, family, pert, 11)
    b = sy.quad_vertices(w, family, pert, 11)
    t = po.TransportOracle(sy.material_s(), w, mesh_family=family, perturbation=pert, mesh_seed=11)
    c = t.vertices()
    assert np.array_equal(bits(a), bits(b)) and np.array_equal(bits(a), bits(c))


def test_mesh_family_checks():
    from mantlepar_b200._capi import MPError
    from mantlepar_b200.transport import mesh_vertices
    w = sy.Workload(nx=4, ny=4)
    with pytest.raises(MPError):
        mesh_vertices(w, 1, 0.25, 1)          # perturbation must be < 0.25
    with pytest.raises(MPError):
        mesh_vertices(w, 5, 0.0, 1)           # unknown family
    assert po.TransportOracle.__init__ is not None
    with pytest.raises(RuntimeError):
        po.TransportOracle(sy.material_s(), w, mesh_family=1, perturbation=0.3)


def test_rectangular_velocities_match_uniform_builder():
    w = sy.Workload(nx=7, ny=5)
    vs, ud = sy.face_velocity_quads(w, sy.quad_vertices(w, 0))
    vs0, ud0 = sy.face_velocity(w)
    assert np.array_equal(vs, vs0) and np.array_equal(ud, ud0)
