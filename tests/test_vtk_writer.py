"""The VTK solution writer against the reference's own: the CPU Euler3D
executable compiled from the reference sources runs a short implicit solve
on a UGRID mesh written by this library and writes its VTK solution and
restart files; cfd_vtk_write, given the same mesh and the restart state,
must produce the identical file (VTK_Writer, Euler3D/src/MeshIO.cpp:219)."""
import subprocess

import numpy as np

from cfdsolutions_b200 import box_mesh, capi, default_params
from cfdsolutions_b200.mesh import write_vtk
from oracle import refharness
from tests._util import make_case, params_from

EXE_CPU = refharness.Path(refharness.__file__).resolve().parent / "_ref" / "euler3d"


def test_vtk_file_is_byte_identical_to_the_reference(ref_available, tmp_path):
    m = box_mesh(5, jitter=0.15, seed=8, with_cells=True, ugrid_path=str(tmp_path / "mesh.ugrid"))
    _, cfg, Q = make_case(mesh=m, seed=8, noise=0.01)
    (tmp_path / "bc.txt").write_text("# number of boundaries\n1\n# boundary 1\n1\n")
    capi.check(capi.lib.cfd_restart_write(str(tmp_path / "in.rst").encode(), 0, m.nnode, m.nghost,
                                          capi.ptr(np.ascontiguousarray(Q))), "restart")
    text = refharness.param_text(cfg)
    text = text.replace("MESH_FILENAME=none", f"MESH_FILENAME={tmp_path / 'mesh.ugrid'}")
    text = text.replace("BC_FILENAME=none", f"BC_FILENAME={tmp_path / 'bc.txt'}")
    text = text.replace("SOLUTION_FILENAME=none", f"SOLUTION_FILENAME={tmp_path / 'ref.vtk'}")
    text = text.replace("SOLVER_NITERATION=1", "SOLVER_NITERATION=2")
    text = text.replace("RESTART_INPUT=NO", f"RESTART_INPUT=YES\nRESTART_INPUT_FILENAME={tmp_path / 'in.rst'}")
    text = text.replace("RESTART_OUTPUT=NO", "RESTART_OUTPUT=YES\nRESTART_OUTPUT_FILENAME=out.rst")
    (tmp_path / "param.txt").write_text(text)
    r = subprocess.run([str(EXE_CPU), str(tmp_path / "param.txt")], cwd=tmp_path, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    Qr = np.empty((5, m.nnode + m.nghost))
    it = __import__("ctypes").c_int()
    capi.check(capi.lib.cfd_restart_read(str(tmp_path / "out.rst").encode(), __import__("ctypes").byref(it),
                                         m.nnode, m.nghost, capi.ptr(Qr)), "restart_read")
    write_vtk(m, tmp_path / "ours.vtk", params_from(cfg), Qr)
    ref, ours = (tmp_path / "ref.vtk").read_bytes(), (tmp_path / "ours.vtk").read_bytes()
    assert len(ref) > 1000
    assert ours == ref


def test_vtk_stiffened_gas_fields(tmp_path):
    """With pinf > 0 the derived fields follow the stiffened gas: a uniform
    water freestream has p = 1, T = (1 + pinf) / (R rho) and its Mach number."""
    m = box_mesh(3, jitter=0.0, seed=1, with_cells=True)
    p = default_params(gamma=4.4, pinf=6000.0, mach=0.0062, mach_min=0.0062, alpha_deg=0.0)
    from cfdsolutions_b200.mesh import perturbed_freestream
    Q = perturbed_freestream(m, 4.4, 0.0062, 0.0, noise=0.0, pinf=6000.0)
    write_vtk(m, tmp_path / "w.vtk", p, Q)
    lines = (tmp_path / "w.vtk").read_text().splitlines()

    def field(name):
        k = lines.index(f"SCALARS {name} double 1")
        return np.array([float(x) for x in lines[k + 2:k + 2 + m.nnode]])

    np.testing.assert_allclose(field("Pressure"), 1.0, rtol=0, atol=1e-10)
    np.testing.assert_allclose(field("Temperature"), 6001.0 * 4.4, rtol=1e-12)
    np.testing.assert_allclose(field("Mach"), 0.0062, rtol=1e-12)


def test_vtk_rup_state_writes_the_conservative_file(tmp_path):
    """A (rho, u, v, w, p) state with variables = CFD_VARS_RUP gives the file
    of the same state in conservative variables (fields to print precision)."""
    from cfdsolutions_b200 import to_rup
    from cfdsolutions_b200.mesh import perturbed_freestream
    m = box_mesh(3, jitter=0.1, seed=1, with_cells=True)
    Q = perturbed_freestream(m, 1.4, 0.5, 2.0, noise=0.02, seed=4)
    write_vtk(m, tmp_path / "c.vtk", default_params(), Q)
    write_vtk(m, tmp_path / "r.vtk", default_params(variables=1), to_rup(Q, 1.4))
    a = (tmp_path / "c.vtk").read_text().splitlines()
    b = (tmp_path / "r.vtk").read_text().splitlines()
    assert len(a) == len(b)
    for x, y in zip(a, b):
        if x != y:
            np.testing.assert_allclose([float(t) for t in y.split()], [float(t) for t in x.split()], rtol=1e-13)
