"""SW2D case files: the writers produce what the readers (the reference's formats) read back."""
import os

import numpy as np

from tests.conftest import load_pkg


def test_case_roundtrip(tmp_path):
    pkg = load_pkg()
    case = pkg.workloads.channel_features(n_cells=600)
    pkg.write_case(str(tmp_path), case)
    back = pkg.read_case(str(tmp_path))
    m, b = case.mesh, back.mesh
    for f in ("cell_area", "cell_x", "cell_y", "cell_z_b", "edge_int_cells", "edge_int_length", "edge_int_nx",
              "edge_int_ny", "edge_int_mx", "edge_int_my", "edge_bnd_cell", "edge_bnd_length", "edge_bnd_nx",
              "edge_bnd_ny", "edge_bnd_code"):
        assert np.array_equal(getattr(m, f), getattr(b, f)), f
    for f in ("h0", "q0", "r0", "phi", "boussinesq", "friction", "head_loss"):
        assert np.array_equal(np.asarray(getattr(case, f)), np.asarray(getattr(back, f))), f
    assert back.bc.codes == case.bc.codes and back.bc.types == case.bc.types
    assert np.array_equal(back.bc.values, case.bc.values)
    assert back.opts["num_scheme"] == "godunov" and back.opts["topo_discretization"] == "blending"


def test_uniform_map(tmp_path):
    pkg = load_pkg()
    p = os.path.join(str(tmp_path), "m.txt")
    pkg.case.write_map(p, ["Kx", "Ky", "alpha"], [60.0, 60.0, 0.0], 5)
    names, arr = pkg.case.read_map(p, 3, 5)
    assert names == ["Kx", "Ky", "alpha"] and arr.shape == (3, 5) and np.all(arr[0] == 60.0)


def test_mesh_orientation():
    """Normals point L -> R on internal edges and into the domain on boundary edges."""
    pkg = load_pkg()
    m = pkg.mesh.jittered_triangle_mesh(12, 7, 10.0, 5.0, seed=3)
    L, R = m.edge_int_cells[:, 0], m.edge_int_cells[:, 1]
    dot = m.edge_int_nx * (m.cell_x[R] - m.cell_x[L]) + m.edge_int_ny * (m.cell_y[R] - m.cell_y[L])
    assert np.all(dot > 0)
    c = m.edge_bnd_cell
    dotb = m.edge_bnd_nx * (m.cell_x[c] - m.edge_bnd_mx) + m.edge_bnd_ny * (m.cell_y[c] - m.edge_bnd_my)
    assert np.all(dotb > 0)
    assert np.isclose(m.cell_area.sum(), 50.0)
    # every cell of a triangle mesh has three edges in all
    cnt = np.bincount(np.concatenate([L, R, c]), minlength=m.cell_nb)
    assert np.all(cnt == 3)
