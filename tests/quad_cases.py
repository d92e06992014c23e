"""Seeded general-quad transport cases (perturbed-quadrilateral and
sine-stretched meshes, src/core/mesh.cpp:27-55) shared by the oracle tests,
the GPU parity tests and the golden-fixture script."""
from __future__ import annotations

from mantlepar_b200 import synthetic as sy


def quad_case(name):
    """Seeded general-quad cases: (workload, family, perturbation, options)."""
    cases = {
        "p12x10": (sy.Workload(nx=12, ny=10, seed=5), 1, 0.2, {}),
        "p3x5": (sy.Workload(nx=3, ny=5, seed=7), 1, 0.24, {}),
        "p9x11_diff": (sy.Workload(nx=9, ny=11, seed=3), 1, 0.15, {"diffusion": True}),
        "s8x7": (sy.Workload(nx=8, ny=7, seed=2, psi_amplitude=0.05), 2, 0.0, {}),
        "p2x2": (sy.Workload(nx=2, ny=2, seed=9), 1, 0.2, {}),
        "p5x4_diff": (sy.Workload(nx=5, ny=4, seed=13, noise_H=0.1), 1, 0.24, {"diffusion": True}),
    }
    return cases[name]


QUAD_CASES = ["p12x10", "p3x5", "p9x11_diff", "s8x7", "p2x2", "p5x4_diff"]


def quad_oracle(name, lib=None, integrator=3):
    """The oracle instance of a case: (handle, vertices, vs_n, ud_n)."""
    from oracle import pyoracle as po
    w, fam, pert, opt = quad_case(name)
    t = po.TransportOracle(sy.material_s(), w, lib=lib, integrator=integrator, mesh_family=fam, perturbation=pert,
                           mesh_seed=11)
    xy = t.vertices()
    vs, ud = sy.face_velocity_quads(w, xy)
    H, C = sy.initial_state(w)
    t.set_face_velocity(vs, ud)
    t.set_state(H, C)
    if opt.get("diffusion"):
        assert t.set_diffusion(0.02, (1, 2, 0, 1), (0.9, -0.02, 0.0, 0.4)) == 0
    return t, xy, vs, ud
