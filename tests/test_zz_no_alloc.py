"""The stage entry point that allocates no device memory.

mp_transport_rhs_noalloc serves callers that cannot call cudaMalloc (code
inside a framework that owns all device memory, or code that must not
allocate once its latency-critical phase has started): all its scratch lives
in a fixed file-scope device array. This test calls it through the C ABI,
twice in a row, and checks both results against the allocating entry point
(mp_transport_rhs through Transport.rhs) with the same tolerance as the other
stage tests; it also checks the stated size limit. It sits in its own file,
collected last, and passes alone in a fresh process as well as after the
other tests.
"""
import ctypes as C

import numpy as np
import pytest

from mantlepar_b200 import synthetic as sy

pytestmark = pytest.mark.gpu
RTOL = 1e-12


def _rel(a, b):
    return np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-3 * max(np.max(np.abs(b)), 1e-300)))


def _rel_inf(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


def _noalloc(w, cfg, H, Cc, vs, ud, with_optional=True):
    """One call of the entry point on device copies of the inputs; with
    with_optional=False the optional rate and totals outputs are NULL."""
    import torch
    from mantlepar_b200 import _capi
    lib = _capi.lib()
    dev = torch.device("cuda", torch.cuda.current_device())
    d = lambda a: torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device=dev)
    Hd, Cd, vd, ud_ = d(H), d(Cc), d(vs), d(ud)
    outs = [torch.empty(w.cells, dtype=torch.float64, device=dev) for _ in range(5)]
    mesh = _capi.MeshDesc(w.nx, w.ny, w.x0, w.x1, w.y0, w.y1)
    opts = cfg.to_c()
    tot = _capi.StageTotals()
    stream = torch.cuda.current_stream(dev).cuda_stream
    ptrs = [o.data_ptr() for o in outs]
    if not with_optional:
        ptrs[4] = None
    code = lib.mp_transport_rhs_noalloc(C.byref(mesh), C.byref(opts), Hd.data_ptr(), Cd.data_ptr(), vd.data_ptr(),
                                        ud_.data_ptr(), *ptrs, C.byref(tot) if with_optional else None, stream)
    _capi.check(code)
    rhsH, rhsC, T, phi, rate = (o.cpu().numpy() for o in outs)
    out = dict(rhsH=rhsH, rhsC=rhsC, T=T, phi=phi)
    if with_optional:
        out.update(rate=rate, maxRate=tot.maxRate, boundaryH=tot.boundaryH, boundaryC=tot.boundaryC)
    return out


# (2, 16384) and (16384, 2) hold the most edges the fixed face region is
# sized for (2.5 * 32768 + 2); (128, 256) is exactly 32768 cells. The two
# skinny meshes take a domain of square cells.
@pytest.mark.parametrize("shape", [(20, 20), (64, 128), (3, 5), (2, 16384), (16384, 2), (128, 256)])
def test_noalloc_stage_matches_allocating_entry_point(shape):
    from mantlepar_b200 import build
    build.build()
    from mantlepar_b200.transport import Transport, TransportConfig
    nx, ny = shape
    skinny = max(nx, ny) >= 16 * min(nx, ny)
    w = sy.Workload(nx=nx, ny=ny, seed=11, x1=(nx / ny if skinny else 0.5))
    cfg = TransportConfig(cfl=w.cfl, integrator=3)
    H, Cc = sy.initial_state(w)
    vs, ud = sy.face_velocity(w)
    ref_t = Transport(w, cfg)
    ref_t.set_face_velocity(vs, ud)
    ref_t.set_state(H, Cc)
    ref = ref_t.rhs()
    ref_t.close()
    first = _noalloc(w, cfg, H, Cc, vs, ud)
    second = _noalloc(w, cfg, H, Cc, vs, ud)
    for got in (first, second):
        for k in ("T", "phi", "rate"):
            assert _rel(got[k], ref[k]) <= RTOL, k
        for k in ("rhsH", "rhsC"):
            assert _rel_inf(got[k], ref[k]) <= RTOL, k
        assert abs(got["maxRate"] - ref["maxRate"]) <= RTOL * ref["maxRate"]
        assert abs(got["boundaryH"] - ref["boundaryH"]) <= RTOL * max(1.0, abs(ref["boundaryH"]))


def test_noalloc_rejects_meshes_above_its_limit():
    from mantlepar_b200 import build
    build.build()
    from mantlepar_b200._capi import MPError
    from mantlepar_b200.transport import TransportConfig
    w = sy.Workload(nx=200, ny=200)          # 40000 cells > 32768
    H, Cc = sy.initial_state(w)
    vs, ud = sy.face_velocity(w)
    with pytest.raises(MPError) as err:
        _noalloc(w, TransportConfig(), H, Cc, vs, ud)
    assert err.value.code == 60


def test_noalloc_optional_outputs_may_be_null():
    """rate and totals may be NULL: the other outputs are unchanged."""
    from mantlepar_b200 import build
    build.build()
    from mantlepar_b200.transport import TransportConfig
    w = sy.Workload(nx=24, ny=40, seed=5)
    cfg = TransportConfig(cfl=w.cfl, integrator=3)
    H, Cc = sy.initial_state(w)
    vs, ud = sy.face_velocity(w)
    full = _noalloc(w, cfg, H, Cc, vs, ud)
    bare = _noalloc(w, cfg, H, Cc, vs, ud, with_optional=False)
    for k in ("rhsH", "rhsC", "T", "phi"):
        assert np.array_equal(full[k], bare[k]), k
