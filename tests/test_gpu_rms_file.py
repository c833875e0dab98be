"""cfd_rms_file_write_ctx: a residual-history line written straight from a
context carries the context's RMS (cfd_residual_rms) and eigenvalue / time
step extrema (cfd_get_extrema) in Euler3D's layout (Euler3D/src/RMSIO.cpp:85-97),
the byte layout itself being pinned by tests/test_rms_file.py."""
import ctypes as C

import numpy as np
import pytest

from cfdsolutions_b200 import Euler3DGPU, capi
from tests._util import make_case, params_from

pytestmark = pytest.mark.gpu


def test_rms_file_line_from_context(gpu_available, tmp_path):
    m, cfg, Q = make_case(n=6, seed=3)
    path = tmp_path / "Residual.res"
    h = C.c_void_p()
    capi.check(capi.lib.cfd_rms_file_open(str(path).encode(), capi.RMSFILE_EULER3D, capi.VARS_CONSERVATIVE, 0,
                                          C.byref(h)), "cfd_rms_file_open")
    with Euler3DGPU(m, params_from(cfg)) as s:
        for it in range(2):
            s.set_state(Q)
            s.begin_iteration(it)
            s.Apply_Boundary_Condition(it)
            s.Compute_Residual(1)
            s.Compute_DeltaT(it)
            capi.check(capi.lib.cfd_rms_file_write_ctx(h, s.handle, it, 0), "cfd_rms_file_write_ctx")
        rms = s.residual_rms(False)
        ext = s.get_extrema()
    capi.check(capi.lib.cfd_rms_file_close(h), "cfd_rms_file_close")
    lines = path.read_text().splitlines()
    assert len(lines) == 4 + 2 + 1 and set(lines[-1]) == {"="}
    vals = np.array([float(x) for x in lines[-2].split()[1:]])
    want = np.r_[rms, ext[6], ext[7], ext[:6]]
    assert int(lines[-2].split()[0]) == 1
    assert np.allclose(vals, want, rtol=6e-6, atol=0.0)
