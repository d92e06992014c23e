"""The C-ABI library builds for sm_100a, loads, and exports every declared symbol."""
import ctypes
import os
import subprocess

from mantlepar_b200 import _capi


def test_header_declares_the_boundary():
    names = _capi.header_functions()
    for n in ["mp_phase_create", "mp_phase_evaluate_batch", "mp_phase_boundaries", "mp_transport_create",
              "mp_transport_set_face_velocity", "mp_transport_set_state", "mp_transport_get_state",
              "mp_transport_rhs", "mp_transport_step", "mp_last_error_string"]:
        assert n in names


def test_library_exports_every_declared_symbol(cuda_lib):
    for n in _capi.header_functions():
        assert hasattr(cuda_lib, n), n
    out = subprocess.run(["nm", "-D", "--defined-only", _capi.LIB_PATH], capture_output=True, text=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    missing = [n for n in _capi.header_functions() if n not in exported]
    assert not missing, missing


def test_build_targets_sm100a_only():
    from mantlepar_b200 import build
    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]
    assert "-lineinfo" in build.FLAGS


def test_host_layer_exports_the_phase_model_interface(cuda_lib):
    """The C++ host layer exports mantle::phase::EutecticModel's members and
    links against the CUDA library (no evaluation without a GPU)."""
    from mantlepar_b200 import build
    assert os.path.exists(build.HOST_LIB)
    out = subprocess.run(["nm", "-DC", "--defined-only", build.HOST_LIB], capture_output=True, text=True).stdout
    for member in ["EutecticModel::EutecticModel(mantle::phase::MaterialParameters const&)",
                   "EutecticModel::evaluate(double, double, double) const",
                   "EutecticModel::classify(double, double, double) const",
                   "EutecticModel::boundaries(double, double) const",
                   "EutecticModel::setParameters(mantle::phase::MaterialParameters const&)",
                   "EutecticModel::pressureCorrectedTemperature(double, double) const",
                   "EutecticModel::staticPressure(double, double) const",
                   "EutecticModel::printInfo(std::ostream&) const"]:
        assert "mantle::phase::" + member in out, member
    deps = subprocess.run(["ldd", build.HOST_LIB], capture_output=True, text=True).stdout
    assert "libmantlepar_b200.so" in deps


def test_invalid_quad_meshes_are_rejected_before_device_work(cuda_lib):
    """mp_transport_create_quads and mp_preheat_create_quads check the vertex
    array on the host (the reference's quad validation) before any device
    call: a null array or a folded cell gives MP_ERR_ARG_WRONG and no handle,
    with no GPU present."""
    import ctypes as C
    import numpy as np
    from mantlepar_b200 import synthetic as sy
    from mantlepar_b200.preheat import PreheatConfig
    from mantlepar_b200.transport import TransportConfig
    w = sy.Workload(nx=4, ny=4)
    mesh = _capi.MeshDesc(w.nx, w.ny, w.x0, w.x1, w.y0, w.y1)
    xy = sy.quad_vertices(w, sy.MESH_RECTANGULAR).reshape(5, 5, 2).copy()
    xy[2, 2] = xy[3, 3] + [0.01, 0.01]            # fold one interior vertex past its neighbour
    bad = np.ascontiguousarray(xy.reshape(-1))
    t_opts, p_opts = TransportConfig().to_c(), PreheatConfig().to_c()
    for xy_ptr in (None, bad.ctypes.data):
        h = C.c_void_p()
        assert cuda_lib.mp_transport_create_quads(C.byref(mesh), xy_ptr, C.byref(t_opts), None, C.byref(h)) == 62
        assert not h.value
        assert cuda_lib.mp_preheat_create_quads(C.byref(mesh), xy_ptr, C.byref(p_opts), None, C.byref(h)) == 62
        assert not h.value
    assert b"quadrilateral" in cuda_lib.mp_last_error_string()


def _noalloc_call(lib, mesh, opts):
    """mp_transport_rhs_noalloc with placeholder (never dereferenced) device
    pointers: every case below is rejected on the host before device work."""
    import ctypes as C
    fake = C.c_void_p(16)
    return lib.mp_transport_rhs_noalloc(C.byref(mesh), C.byref(opts), fake, fake, fake, fake, fake, fake, fake, fake,
                                        None, None, None)


def test_noalloc_checks_options_as_the_allocating_entry_points(cuda_lib):
    """One options struct is rejected alike by mp_transport_create,
    mp_batch_create and mp_transport_rhs_noalloc: bad boundary policies and
    an inflow composition outside [0, Xe] give MP_ERR_ARG_OUTOFRANGE from
    each, before any device call (no GPU is present here)."""
    import ctypes as C
    import dataclasses
    from mantlepar_b200 import synthetic as sy
    from mantlepar_b200.transport import TransportConfig
    w = sy.Workload(nx=8, ny=8)
    mesh = _capi.MeshDesc(w.nx, w.ny, w.x0, w.x1, w.y0, w.y1)
    base = TransportConfig(cfl=0.4, integrator=3)
    bad = [dataclasses.replace(base, H_policy=3), dataclasses.replace(base, C_policy=-1),
           dataclasses.replace(base, inflow_C=0.6), dataclasses.replace(base, inflow_C=-0.1),
           dataclasses.replace(base, cfl=1.5), dataclasses.replace(base, integrator=4),
           dataclasses.replace(base, precision=7)]
    for cfg in bad:
        opts = cfg.to_c()
        h = C.c_void_p()
        c_create = cuda_lib.mp_transport_create(C.byref(mesh), C.byref(opts), None, C.byref(h))
        c_batch = cuda_lib.mp_batch_create(C.byref(mesh), 1, C.byref(opts), None, C.byref(h))
        c_noalloc = _noalloc_call(cuda_lib, mesh, opts)
        assert c_create == c_batch == c_noalloc == 63, (cfg, c_create, c_batch, c_noalloc)
        assert not h.value


def test_noalloc_rejects_unsupported_options_on_the_host(cuda_lib):
    """Thermal diffusion, the adiabatic source and the mixed-precision form
    are not evaluated by mp_transport_rhs_noalloc: MP_ERR_ARG_WRONG, with a
    message naming the entry point; a mesh above 32768 cells: MP_ERR_ARG_SIZ."""
    import dataclasses
    from mantlepar_b200 import synthetic as sy
    from mantlepar_b200.transport import TransportConfig
    w = sy.Workload(nx=8, ny=8)
    mesh = _capi.MeshDesc(w.nx, w.ny, w.x0, w.x1, w.y0, w.y1)
    base = TransportConfig(cfl=0.4, integrator=3)
    for cfg in (dataclasses.replace(base, diffusivity=1e-4),
                dataclasses.replace(base, material=dataclasses.replace(sy.material_s(), alpha0=3e-5)),
                dataclasses.replace(base, precision=1)):
        assert _noalloc_call(cuda_lib, mesh, cfg.to_c()) == 62
        assert b"mp_transport_rhs_noalloc" in cuda_lib.mp_last_error_string()
    big = _capi.MeshDesc(2, 16385, w.x0, w.x1, w.y0, w.y1)
    assert _noalloc_call(cuda_lib, big, base.to_c()) == 60


def test_checked_variant_exports_the_same_symbols(cuda_lib):
    """The bounds-checked build (MP_CHECKED) exports every declared symbol too."""
    from mantlepar_b200 import build
    path = build.build_checked()
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    missing = [n for n in _capi.header_functions() if n not in exported]
    assert not missing, missing


def test_transport_instance_bytes_is_host_arithmetic(cuda_lib):
    """mp_transport_instance_bytes (the serving budget of a quad-mesh request)
    needs no device: 0 for an invalid mesh, the per-cell tables of a quad mesh
    on top of the uniform transport's arrays, and growth with the cell count."""
    import ctypes as C
    lib = _capi.lib()
    def nbytes(nx, ny, quads):
        return lib.mp_transport_instance_bytes(C.byref(_capi.MeshDesc(nx, ny, 0.0, 0.5, 0.0, 1.0)), quads)
    assert nbytes(1, 8, 0) == 0 and nbytes(8, 1, 1) == 0
    u, q = nbytes(256, 512, 0), nbytes(256, 512, 1)
    assert 0 < u < q
    assert (q - u) / (256 * 512) > 184 * 8     # per-cell tables: 184 doubles a cell
    assert nbytes(512, 1024, 1) > 3.5 * q      # whole 2 MiB pages per allocation
    assert u % (2 << 20) == 0 and q % (2 << 20) == 0
