"""Drop-in test: the reference's own Euler3D executable, once as compiled
from its sources (CPU) and once with its hot-path functions taken from the
CUDA library through cfdsolutions_b200/csrc/euler3d_shim.cpp, run the same
UGRID mesh, boundary-condition file, parameter file and perturbed restart
state (Euler3D/main.cpp:94-160, Solver_Steady_Implicit.cpp:35-184).  Their
residual histories (Residual.res) and final restart states must agree."""
import os
import subprocess
from pathlib import Path

import numpy as np
import pytest

from cfdsolutions_b200 import box_mesh, capi
from oracle import refharness
from tests._util import make_case

pytestmark = pytest.mark.gpu

REF_DIR = Path(refharness.__file__).resolve().parent / "_ref"
EXE_CPU = REF_DIR / "euler3d"
EXE_GPU = REF_DIR / "euler3d_gpu"


def write_case(d: Path, n: int, order: int, iters: int, seed: int = 5, jacobian_method: int = 4, flux: int = 0):
    m = box_mesh(n, jitter=0.15, seed=seed, ugrid_path=str(d / "mesh.ugrid"))
    _, cfg, Q = make_case(mesh=m, noise=0.01)
    (d / "bc.txt").write_text("# number of boundaries\n1\n# boundary 1\n1\n")
    rst = str(d / "in.rst").encode()
    capi.check(capi.lib.cfd_restart_write(rst, 0, m.nnode, m.nghost, capi.ptr(np.ascontiguousarray(Q))), "restart")
    cfg = dict(cfg, order=order, limiter=1 if order else -1, venkat_k=5.0, jacobian_method=jacobian_method,
               flux_scheme=flux)
    text = refharness.param_text(cfg)
    text = text.replace("MESH_FILENAME=none", f"MESH_FILENAME={d / 'mesh.ugrid'}")
    text = text.replace("BC_FILENAME=none", f"BC_FILENAME={d / 'bc.txt'}")
    text = text.replace("SOLUTION_FILENAME=none", f"SOLUTION_FILENAME={d / 'sol.vtk'}")
    text = text.replace("SOLVER_NITERATION=1", f"SOLVER_NITERATION={iters}")
    text = text.replace("RESTART_INPUT=NO", f"RESTART_INPUT=YES\nRESTART_INPUT_FILENAME={d / 'in.rst'}")
    text = text.replace("RESTART_OUTPUT=NO", "RESTART_OUTPUT=YES\nRESTART_OUTPUT_FILENAME=out.rst")
    (d / "param.txt").write_text(text)
    return m


def run(exe: Path, d: Path, param: Path):
    d.mkdir(exist_ok=True)
    r = subprocess.run([str(exe), str(param)], cwd=d, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    rows = [list(map(float, ln.split())) for ln in (d / "Residual.res").read_text().splitlines()
            if ln.strip() and ln.strip()[0].isdigit()]
    raw = (d / "out.rst").read_bytes()
    return np.array(rows), raw


@pytest.mark.parametrize("order,flux", [(0, 0), (1, 0), (1, 3)])
def test_euler3d_executable_with_gpu_hot_path(gpu_available, ref_available, tmp_path, order, flux):
    """flux 3: Roe with the low-Mach fix (PRECOND_METHOD_ROE_LMFIX)."""
    if not EXE_GPU.exists():
        pytest.skip("drop-in executable not built (make -C oracle gpu)")
    iters = 6
    m = write_case(tmp_path, 8, order, iters, flux=flux)
    res_cpu, rst_cpu = run(EXE_CPU, tmp_path / "cpu", tmp_path / "param.txt")
    res_gpu, rst_gpu = run(EXE_GPU, tmp_path / "gpu", tmp_path / "param.txt")
    assert res_cpu.shape == res_gpu.shape and res_cpu.shape[0] == iters
    # Residual.res prints 6 significant digits (%10.5e)
    np.testing.assert_allclose(res_gpu, res_cpu, rtol=2e-5, atol=0)
    hdr_c, hdr_g = np.frombuffer(rst_cpu[:16], np.int32), np.frombuffer(rst_gpu[:16], np.int32)
    np.testing.assert_array_equal(hdr_c, hdr_g)
    qc = np.frombuffer(rst_cpu[16:], np.float64)
    qg = np.frombuffer(rst_gpu[16:], np.float64)
    assert np.abs(qg - qc).max() <= 1e-10 * np.abs(qc).max()


@pytest.mark.parametrize("method,flux", [("TIME_INTEGRATION_METHOD_EXPLICIT_EULER", 0),
                                         ("TIME_INTEGRATION_METHOD_EXPLICIT_RK4", 0),
                                         ("TIME_INTEGRATION_METHOD_EXPLICIT_RK4", 6)])
def test_euler3d_explicit_executable_with_gpu_hot_path(gpu_available, ref_available, tmp_path, method, flux):
    """The reference's explicit drivers (Solver_Steady_Explicit_Euler / _RK4,
    Euler3D/src/Solver_Steady_Explicit.cpp:25, :202) over the GPU residual,
    gradient, limiter, boundary and time-step functions; flux 6 is
    FLUX_SCHEME_VANLEER, which the reference runs with its explicit drivers only."""
    if not EXE_GPU.exists():
        pytest.skip("drop-in executable not built (make -C oracle gpu)")
    iters = 5
    write_case(tmp_path, 8, 1, iters, flux=flux)
    text = (tmp_path / "param.txt").read_text()
    text = text.replace("SOLVER_SCHEME=SOLVER_SCHEME_IMPLICIT", "SOLVER_SCHEME=SOLVER_SCHEME_EXPLICIT")
    text = text.replace("TIME_INTEGRATION_METHOD=TIME_INTEGRATION_METHOD_IMPLICIT_EULER", f"TIME_INTEGRATION_METHOD={method}")
    text = text.replace("CFL_MIN=10.0", "CFL_MIN=1.0").replace("CFL_MAX=10.0", "CFL_MAX=1.0")  # explicit stability
    assert "SOLVER_SCHEME_EXPLICIT" in text and method in text
    (tmp_path / "param.txt").write_text(text)
    res_cpu, rst_cpu = run(EXE_CPU, tmp_path / "cpu", tmp_path / "param.txt")
    res_gpu, rst_gpu = run(EXE_GPU, tmp_path / "gpu", tmp_path / "param.txt")
    assert res_cpu.shape == res_gpu.shape and res_cpu.shape[0] == iters
    np.testing.assert_allclose(res_gpu, res_cpu, rtol=2e-5, atol=0)
    qc = np.frombuffer(rst_cpu[16:], np.float64)
    qg = np.frombuffer(rst_gpu[16:], np.float64)
    assert np.abs(qg - qc).max() <= 1e-10 * np.abs(qc).max()


def test_euler3d_unsteady_executable_with_gpu_hot_path(gpu_available, ref_available, tmp_path):
    """The reference's physical-time driver (Solver_Unsteady_Implicit,
    Euler3D/src/Solver_Unsteady_Implicit.cpp:41, BDF2, 3 steps x 3 inner
    iterations) edits the host block system between Compute_Jacobian and the
    block sweeps; the shim mirrors the system to the host and back for it."""
    if not EXE_GPU.exists():
        pytest.skip("drop-in executable not built (make -C oracle gpu)")
    write_case(tmp_path, 6, 0, 3)
    text = (tmp_path / "param.txt").read_text()
    text = text.replace("SOLVER_METHOD=SOLVER_METHOD_STEADY", "SOLVER_METHOD=SOLVER_METHOD_UNSTEADY")
    text = text.replace("TIME_INTEGRATION_METHOD=TIME_INTEGRATION_METHOD_IMPLICIT_EULER",
                        "TIME_INTEGRATION_METHOD=TIME_INTEGRATION_METHOD_IMPLICIT_EULER_BDF")
    text += "\nPHYSICAL_DELTA_TIME=0.05\nSOLVER_INNER_NITERATION=3\n"
    (tmp_path / "param.txt").write_text(text)
    res_cpu, rst_cpu = run(EXE_CPU, tmp_path / "cpu", tmp_path / "param.txt")
    res_gpu, rst_gpu = run(EXE_GPU, tmp_path / "gpu", tmp_path / "param.txt")
    assert res_cpu.shape == res_gpu.shape and res_cpu.shape[0] == 9
    np.testing.assert_allclose(res_gpu, res_cpu, rtol=2e-5, atol=0)
    qc = np.frombuffer(rst_cpu[16:], np.float64)
    qg = np.frombuffer(rst_gpu[16:], np.float64)
    assert np.abs(qg - qc).max() <= 1e-10 * np.abs(qc).max()


def test_euler3d_executable_gmres_converges(gpu_available, ref_available, tmp_path):
    """Same executable with the block sweeps replaced by mixed-precision
    GMRES(30)+ILU(0) (CFD_B200_LINEAR=gmres): the residual still drops.
    (Euler3D's right-hand side leaves out the dissipative residual,
    FluxTest.cpp:8143-8150, so its implicit iterations converge slowly with any
    linear solver; the CPU block Gauss-Seidel run drops ~30% in 6 iterations.)"""
    if not EXE_GPU.exists():
        pytest.skip("drop-in executable not built (make -C oracle gpu)")
    write_case(tmp_path, 8, 0, 8)
    d = tmp_path / "gmres"
    d.mkdir()
    env = dict(os.environ, CFD_B200_LINEAR="gmres")
    r = subprocess.run([str(EXE_GPU), str(tmp_path / "param.txt")], cwd=d, capture_output=True, text=True,
                       timeout=600, env=env)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    rows = [list(map(float, ln.split())) for ln in (d / "Residual.res").read_text().splitlines()
            if ln.strip() and ln.strip()[0].isdigit()]
    rms = np.array(rows)[:, 6]
    assert rms[-1] < 0.8 * rms[0]


def test_euler3d_executable_with_finite_difference_jacobian(gpu_available, ref_available, tmp_path):
    """JACOBIAN_METHOD_CENTRAL: the executable's Compute_Jacobian runs the GPU
    finite-difference Jacobian.  Its boundary blocks are difference quotients
    through ghost states that differ from the reference's in the last bits, so
    the states agree to 1e-9 rather than 1e-10."""
    if not EXE_GPU.exists():
        pytest.skip("drop-in executable not built (make -C oracle gpu)")
    iters = 4
    write_case(tmp_path, 6, 0, iters, jacobian_method=0)
    res_cpu, rst_cpu = run(EXE_CPU, tmp_path / "cpu", tmp_path / "param.txt")
    res_gpu, rst_gpu = run(EXE_GPU, tmp_path / "gpu", tmp_path / "param.txt")
    assert res_cpu.shape == res_gpu.shape and res_cpu.shape[0] == iters
    np.testing.assert_allclose(res_gpu, res_cpu, rtol=2e-5, atol=0)
    qc = np.frombuffer(rst_cpu[16:], np.float64)
    qg = np.frombuffer(rst_gpu[16:], np.float64)
    assert np.abs(qg - qc).max() <= 1e-9 * np.abs(qc).max()
