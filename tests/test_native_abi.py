"""CPU-side checks of the C ABI: the library loads, exports every entry point
include/dioptrin_gpu.h declares, and rejects bad configurations before it
touches a device (src/integration/cuda.rs:1071-1088 gives that order)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = []
    for f in os.listdir(os.path.join(ROOT, "include")):
        if f.endswith(".h"):
            text = open(os.path.join(ROOT, "include", f)).read()
            names += re.findall(r"DG_EXPORT\s+[\w\s\*]+?\b(dg_\w+)\s*\(", text)
    return sorted(set(names))


@pytest.fixture(scope="module")
def native():
    from dioptrin_b200 import build, _native
    build.build()
    return _native


def test_every_declared_symbol_is_exported(native):
    names = declared_symbols()
    assert len(names) >= 17
    lib = native.lib()
    for n in names:
        assert hasattr(lib, n), n
    assert sorted(native.EXPORTS) == names


def test_only_the_c_abi_is_exported(native):
    import subprocess
    out = subprocess.run(["nm", "-D", "--defined-only", native.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = sorted(l.split()[-1] for l in out.splitlines() if " T " in l)
    assert exported == declared_symbols()


def _integrator(**kw):
    import dioptrin_b200 as d
    return d.Integrator.from_poni_dict(dict(pixel1=1e-4, pixel2=1e-4, distance=0.1,
                                            poni1=1e-3, poni2=1e-3, wavelength=1e-10), **kw)


def test_configuration_errors_come_before_the_device(native):
    it = _integrator()
    with pytest.raises(ValueError, match="n_points"):
        it.prepare_cuda1d((10, 10), 0)
    with pytest.raises(ValueError, match="zero side"):
        it.prepare_cuda1d((0, 10), 10)
    with pytest.raises(ValueError):
        it.prepare_cuda1d((10, 10), 10, precision="f16")
    with pytest.raises(ValueError):
        it.prepare_cuda1d((10, 10), 10, max_batch_bytes=0)
    with pytest.raises(OverflowError):
        it.prepare_cuda1d((10, 10), 10, device=-1)
    it.set_mask(np.zeros((5, 5), np.uint8))
    with pytest.raises(ValueError, match="mask shape"):
        it.prepare_cuda1d((10, 10), 10)


def test_integrator_option_validation():
    with pytest.raises(ValueError):
        _integrator(method="histogram")
    with pytest.raises(ValueError):
        _integrator(polarization_factor=1.5)
    with pytest.raises(ValueError):
        _integrator(unit="q_mm^-1")
    with pytest.raises(ValueError):
        _integrator(radial_range=(2.0, 1.0))
    with pytest.raises(ValueError):
        _integrator(method="supersampled", n_ss=0)
    with pytest.raises(ValueError):
        _integrator(mask_mode="sometimes")
    it = _integrator()
    with pytest.raises(TypeError):
        it.batch1d("frame.tif", 10)
    with pytest.raises(TypeError):
        it.batch1d_iter("frame.tif", 10)


def test_c_level_argument_checks(native):
    L = native.lib()
    assert L.dg_plan_create(None, None, None, 1, 1, 1, 0, None, None) == native.DG_INVALID_INPUT
    assert "NULL" in native.last_error()
    assert L.dg_integrate(None, None, 1, 1, 0, None, None, None) == native.DG_INVALID_INPUT
    assert L.dg_plan_destroy(None) == native.DG_OK
    g, m = native.Geometry(), native.Method()
    m.kind = 1
    out = C.c_void_p()
    assert L.dg_plan_create(C.byref(g), C.byref(m), None, 4, 4, 8, -1, None,
                            C.byref(out)) == native.DG_INVALID_INPUT
    m.kind = 9
    assert L.dg_plan_create(C.byref(g), C.byref(m), None, 4, 4, 8, 0, None,
                            C.byref(out)) == native.DG_UNSUPPORTED


def test_no_device_raises_unavailable(native):
    import dioptrin_b200 as d
    if d.cuda_available():
        pytest.skip("a device is present")
    info = d.cuda_info()
    assert info["compiled"] and not info["available"] and info["reason"]
    with pytest.raises(d.CudaUnavailableError):
        _integrator().prepare_cuda1d((10, 10), 10)
    with pytest.raises(d.CudaUnavailableError):
        d.RequestLoop()


def test_poni_files_parse(tmp_path):
    from dioptrin_b200 import Poni
    v1 = tmp_path / "v1.poni"
    v1.write_text("# c\nPixelSize1: 0.000172\nPixelSize2: 0.000172\nDistance: 0.2\n"
                  "Poni1: 0.08\nPoni2: 0.07\nRot1: 0.01\nRot2: 0\nRot3: 0\nWavelength: 4e-11\n")
    p = Poni.load(str(v1))
    assert (p.pixel1, p.distance, p.rot1, p.wavelength) == (0.000172, 0.2, 0.01, 4e-11)
    v2 = tmp_path / "v2.poni"
    v2.write_text('poni_version: 2\nDetector: Detector\nDetector_config: {"pixel1": 0.0002, '
                  '"pixel2": 0.0003, "max_shape": [605, 1070]}\nDistance: 0.35\nPoni1: -0.05\n'
                  "Poni2: 0.14\nRot1: 0\nRot2: 0\nRot3: 0\nWavelength: 6.858e-11\n")
    p = Poni.load(str(v2))
    assert (p.pixel1, p.pixel2, p.poni1) == (0.0002, 0.0003, -0.05)
