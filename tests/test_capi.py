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
