"""Seeded preheat cases shared by the oracle tests, the GPU parity tests and
the golden-fixture script: the synthetic streamfunction flow plus an optional
uniform upward through-flow (inflow at the bottom wall, outflow at the top),
thermal diffusion with per-wall conditions, and the step controls of the
reference's input (time.end, control, initial/minimum/maximum step, cfl)."""
from __future__ import annotations

import dataclasses

import numpy as np

from mantlepar_b200 import synthetic as sy


@dataclasses.dataclass
class PreheatCase:
    w: sy.Workload
    through: float = 0.0                      # upward through-flow speed
    bottom_outflow: float = 0.0               # outward speed through the bottom wall only
    kappa: float = 0.0
    thermal_type: tuple = (0, 0, 0, 0)        # walls bottom, top, left, right
    thermal_value: tuple = (0.0, 0.0, 0.0, 0.0)
    H_policy: int = 0
    inflow_H: float = 0.8
    lf_global: int = 0
    lf_global_speed: float = 0.0
    control: int = 0                          # 0 cfl, 1 fixed
    end: float = 0.05
    max_steps: int = 100000
    dt_initial: float = 1e-3
    dt_min: float = 1e-9
    dt_max: float = 1e-2
    cfl: float = 0.5
    pressure_model: int = 0                   # 0 constant (0 Pa), 1 lithostatic
    surface_y: float = 1.1
    family: int = 0                           # MESH_RECTANGULAR / PERTURBED / SINE
    perturbation: float = 0.0
    mesh_seed: int = 11

    def vertices(self):
        """Vertices of a general quad mesh (None on the uniform mesh)."""
        if self.family == sy.MESH_RECTANGULAR:
            return None
        return sy.quad_vertices(self.w, self.family, self.perturbation, self.mesh_seed)

    def velocity(self) -> np.ndarray:
        """Normal Stokes velocity at the edge Gauss points, [edge, q]."""
        nI = self.w.nx * (self.w.ny + 1)
        if self.family != sy.MESH_RECTANGULAR:
            # The through-flow (0, through) against each edge's own normal.
            vs, ud = sy.face_velocity_quads(self.w, self.vertices())
            vs = vs + self.through * (ud / self.w.darcy)
            vs[:self.w.nx] += self.bottom_outflow
            return np.ascontiguousarray(vs)
        vs, _ = sy.face_velocity(self.w)
        vs = vs.copy()
        vs[:nI] += -self.through                # upward: v . (0, -1)
        vs[:self.w.nx] += self.bottom_outflow   # bottom wall: (0, -1) is outward
        return np.ascontiguousarray(vs)

    def state(self):
        return sy.initial_state(self.w)


CASES = {
    "closed": PreheatCase(sy.Workload(nx=12, ny=10, seed=5, noise_H=0.1)),
    "through_diffusion": PreheatCase(sy.Workload(nx=7, ny=9, seed=3), through=0.3, kappa=2e-3,
                                     thermal_type=(1, 1, 0, 2), thermal_value=(1.2, 0.1, 0.0, 0.05)),
    "global_fixed": PreheatCase(sy.Workload(nx=9, ny=8, seed=11), through=0.1, kappa=1e-3, lf_global=1,
                                lf_global_speed=1.5, control=1, dt_initial=4e-3, end=0.03,
                                thermal_type=(2, 1, 1, 0), thermal_value=(-0.02, 0.3, 0.7, 0.0),
                                pressure_model=1),
    "tiny_2x2": PreheatCase(sy.Workload(nx=2, ny=2, seed=4), through=0.2, kappa=3e-3, end=0.02,
                            thermal_type=(1, 2, 1, 0), thermal_value=(1.0, -0.01, 0.5, 0.0)),
    # General quad meshes (the reference's preheat reads every face's and
    # cell's own corners, preheat.cpp:86-117).
    "quad_through": PreheatCase(sy.Workload(nx=9, ny=7, seed=3), through=0.3, kappa=2e-3,
                                thermal_type=(1, 1, 0, 2), thermal_value=(1.2, 0.1, 0.0, 0.05),
                                family=sy.MESH_PERTURBED, perturbation=0.2),
    "quad_sine_fixed": PreheatCase(sy.Workload(nx=8, ny=6, seed=11), through=0.1, kappa=1e-3, lf_global=1,
                                   lf_global_speed=1.5, control=1, dt_initial=1e-3, end=0.006,
                                   thermal_type=(2, 1, 1, 0), thermal_value=(-0.02, 0.3, 0.7, 0.0),
                                   pressure_model=1, family=sy.MESH_SINE_STRETCHED),
    "quad_outflow": PreheatCase(sy.Workload(nx=6, ny=9, seed=21, noise_H=0.08), bottom_outflow=0.2, kappa=5e-4,
                                H_policy=1, thermal_type=(1, 0, 2, 2), thermal_value=(0.4, 0.0, 0.01, -0.01),
                                end=0.02, family=sy.MESH_PERTURBED, perturbation=0.24),
    "quad_2x2": PreheatCase(sy.Workload(nx=2, ny=2, seed=8), through=0.2, kappa=3e-3, end=0.02,
                            thermal_type=(1, 2, 1, 0), thermal_value=(1.0, -0.01, 0.5, 0.0),
                            family=sy.MESH_PERTURBED, perturbation=0.2),
}


def oracle_instance(case: PreheatCase, lib=None):
    """A transport oracle handle set up for the preheat of `case`."""
    from oracle import pyoracle as po
    t = po.TransportOracle(sy.material_s(), case.w, lib=lib, H_policy=case.H_policy, inflow_H=case.inflow_H,
                           lf_global=case.lf_global, lf_global_speed=case.lf_global_speed, cfl=case.cfl,
                           dt_initial=case.dt_initial, dt_max=case.dt_max, dt_min=case.dt_min,
                           mesh_family=case.family, perturbation=case.perturbation, mesh_seed=case.mesh_seed)
    if case.family != sy.MESH_RECTANGULAR:
        assert np.array_equal(t.vertices(), case.vertices())
    vs = case.velocity()
    t.set_face_velocity(vs, np.zeros_like(vs))
    H, C = case.state()
    t.set_state(H, C)
    assert t.set_diffusion(case.kappa, case.thermal_type, case.thermal_value) == 0
    assert t.set_time_control(case.control, case.end) == 0
    if case.pressure_model == 1:
        assert t.set_pressure_model(1, case.surface_y) == 0
    return t


def oracle_run(case: PreheatCase, lib=None) -> dict:
    """begin, rhs, the whole run and the diagnostics on the oracle."""
    t = oracle_instance(case, lib)
    code, rate, limit, first = t.preheat_begin()
    out = dict(begin=code, rate=rate, limit=limit, first=first)
    code, rhs, bflux = t.preheat_rhs()
    out.update(rhs_code=code, rhs=rhs, bflux=bflux)
    code, rows = out["begin"], []
    while code == 0:
        code, got = t.preheat_advance(1000, case.max_steps)
        rows += got
        if len(got) < 1000:
            break
    out.update(run=code, rows=rows, H=t.get_state()[0])
    code, T, phi = t.preheat_diagnostics()
    out.update(diag=code, T=T, phi=phi)
    return out


def gpu_config(case: PreheatCase):
    from mantlepar_b200.preheat import PreheatConfig
    return PreheatConfig(material=sy.material_s(), pressure_model=case.pressure_model,
                         pressure=case.surface_y if case.pressure_model == 1 else 0.0, end=case.end,
                         max_steps=case.max_steps, control=case.control, dt_initial=case.dt_initial,
                         dt_min=case.dt_min, dt_max=case.dt_max, cfl=case.cfl, diffusivity=case.kappa,
                         thermal_type=case.thermal_type, thermal_value=case.thermal_value, H_policy=case.H_policy,
                         inflow_H=case.inflow_H, lf_global=case.lf_global, lf_global_speed=case.lf_global_speed)


def gpu_instance(case: PreheatCase):
    from mantlepar_b200.preheat import Preheat
    p = Preheat(case.w, gpu_config(case), vertices=case.vertices())
    p.set_velocity(case.velocity())
    H, C = case.state()
    p.set_state(H, C)
    return p
