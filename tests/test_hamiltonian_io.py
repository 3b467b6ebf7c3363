"""The grid Hamiltonian file (Hmt.xml / Hmt.json) through the C ABI (a43g_hamiltonian_*), no GPU:
the layouts of the reference's writer (include/grid_operators.hxx:460-613) read back exactly in
both formats, documents in that layout written by hand (comments, self-closing elements, the
reference's exact-zero abbreviation, missing potential values) read as the reference's loaders
read them (src/green_input.cxx:29-221, include/json_reading.hxx:61-229), errors reported, and a
plan built from a file identical to the plan built from the same arrays (with the positions as
the writer rounds them)."""
import numpy as np
import pytest

from angstromcube_b200 import green_function as gf, green_input, workloads


def grid_potential(w):
    """[nz, ny, nx] potential of a workload (its [ncells][64] cubes unfolded)."""
    ng = np.array(w.geometry.ng)
    nb = ng // 4
    return w.Vcell.reshape(nb[2], nb[1], nb[0], 4, 4, 4).transpose(0, 3, 1, 4, 2, 5).reshape(ng[2], ng[1], ng[0])


def workload_arrays(name="periodic8_8atoms_s2x2x1"):
    w = workloads.make(name)
    g = w.geometry
    mats = []
    for a in range(w.natoms):
        n = workloads.nsho(int(g.xyzZinso[a, 5]))
        mats.append(w.mats[w.offsets[a]:w.offsets[a] + 2 * n * n].reshape(2, n, n))
    return w, g, grid_potential(w), mats


@pytest.mark.parametrize("fmt", ["xml", "json"])
def test_write_and_read_back(tmp_path, fmt):
    w, g, V, mats = workload_arrays()
    f = tmp_path / ("Hmt." + fmt)
    green_input.write_to_file(f, g.ng, g.bc, g.hg, V, g.xyzZinso, mats, fileformat=fmt, spectrum=[-1.0, 2.0, 0.1])
    ng, bc, hg, V2, na, xyz, mats2 = green_input.load_Hamiltonian(f)
    assert tuple(ng) == tuple(g.ng) and tuple(bc) == tuple(g.bc) and np.allclose(hg, g.hg, rtol=0, atol=1e-16)
    assert na == w.natoms
    # %.15f potential, %.12f positions, %.15e matrices: the writer's digits
    assert np.abs(V2 - V).max() <= 1e-15
    assert np.abs(xyz[:, :3] - g.xyzZinso[:, :3]).max() <= 1e-12
    assert np.array_equal(xyz[:, 5], g.xyzZinso[:, 5]) and np.allclose(xyz[:, 6], g.xyzZinso[:, 6], atol=1e-12)
    for m, m2 in zip(mats, mats2):
        assert np.abs(m - m2).max() <= 1e-15 * np.abs(m).max()


HAND_WRITTEN = """<?xml version="1.0"?>
<grid_Hamiltonian version="0.0">
  <!-- a comment -->
  <sho_atoms number="1">
    <atom global_id="7" Z="13">
      <position x="0.25" y="-0.5" z="1.125" unit="Bohr"/>
      <projectors type="sho" numax="1" sigma="0.75" unit="Bohr"/>
      <hamiltonian unit="Hartree">
         1.5e-01 2.0e-02 0 0
         2.0e-02 -3.0e-01 0 0
         0 0 4.0e-01 1.0e-03
         0 0 1.0e-03 4.0e-01
      </hamiltonian>
      <overlap unit="1">
         1 0 0 0
         0 1 0 0
         0 0 1 0
         0 0 0 1
      </overlap>
    </atom>
  </sho_atoms>
  <spacing x="0.25" y="0.25" z="0.5" unit="Bohr"/>
  <boundary x="1" y="0" z="2"/>
  <potential nx="4" ny="4" nz="4" unit="Hartree">
    0.5 0.25 -1.0
  </potential>
</grid_Hamiltonian>
"""


def test_read_hand_written_xml(tmp_path):
    f = tmp_path / "Hmt.xml"
    f.write_text(HAND_WRITTEN)
    ng, bc, hg, V, na, xyz, mats = green_input.load_Hamiltonian(f)
    assert tuple(ng) == (4, 4, 4) and tuple(bc) == (1, 0, 2) and tuple(hg) == (0.25, 0.25, 0.5)
    # missing potential values are zero (the reference's default, +green_input.empty.potential=1)
    assert V.shape == (4, 4, 4) and V.ravel()[:3].tolist() == [0.5, 0.25, -1.0] and not V.ravel()[3:].any()
    assert na == 1 and xyz[0].tolist() == [0.25, -0.5, 1.125, 13, 7, 1, 0.75, 0]
    assert mats[0].shape == (2, 4, 4) and mats[0][0, 0, 1] == 0.02 and np.array_equal(mats[0][1], np.eye(4))


def test_read_hand_written_json(tmp_path):
    f = tmp_path / "Hmt.json"
    f.write_text('{"comment": "test", "spacing": [0.5, 0.5, 0.5], "boundary": [1, 1, 1],'
                 ' "potential": {"grid": [4, 4, 4], "values": [1, 2, 3]},'
                 ' "sho_atoms": {"number": 1, "atoms": [{"atom_id": 3, "Z": 6, "position": [0.1, 0.2, 0.3],'
                 ' "projectors": {"type": "sho", "numax": 0, "sigma": 0.5},'
                 ' "hamiltonian": [[0.25]], "overlap": [[1.5]]}]}}')
    ng, bc, hg, V, na, xyz, mats = green_input.load_Hamiltonian(f)
    assert tuple(ng) == (4, 4, 4) and tuple(bc) == (1, 1, 1) and tuple(hg) == (0.5, 0.5, 0.5)
    assert V.ravel()[:4].tolist() == [1, 2, 3, 0]
    # as the reference's JSON loader: Z is not taken from the file
    assert na == 1 and xyz[0].tolist() == [0.1, 0.2, 0.3, 0, 3, 0, 0.5, 0]
    assert mats[0][0, 0, 0] == 0.25 and mats[0][1, 0, 0] == 1.5


def test_bad_documents_are_errors(tmp_path):
    f = tmp_path / "Hmt.xml"
    f.write_text(HAND_WRITTEN.replace("</overlap>", ""))
    with pytest.raises(RuntimeError, match="end tag"):
        green_input.load_Hamiltonian(f)
    f.write_text(HAND_WRITTEN.replace("0 0 0 1\n      </overlap>", "0 0 0\n      </overlap>"))
    with pytest.raises(RuntimeError, match="overlap matrix"):
        green_input.load_Hamiltonian(f)
    with pytest.raises(RuntimeError, match="cannot read"):
        green_input.load_Hamiltonian(tmp_path / "missing.xml")


def test_plan_from_file_equals_plan_from_arrays(tmp_path):
    w, g, V, mats = workload_arrays()
    f = tmp_path / "Hmt.xml"
    green_input.write_to_file(f, g.ng, g.bc, g.hg, V, g.xyzZinso, mats)
    geo, Vg, flat, offs = green_input.geometry_from_file(f, r_trunc=g.r_trunc, sources=g.sources, nFD=g.nFD)
    p1 = gf.construct_Green_function(geo)
    gf.update_potential(p1, Vg, flat, offs, layout="grid")
    gf.update_energy_parameter(p1, w.E, w.dVol)
    # the same cell from the arrays, with the positions as the file holds them (%.12f)
    _, _, _, _, _, xyz, _ = green_input.load_Hamiltonian(f)
    g0 = workloads.Geometry(g.ng, g.bc, g.hg, g.r_trunc, g.sources, g.nFD, g.proj_radius, g.xyzZinso.copy())
    g0.xyzZinso[:, :3] = xyz[:, :3]
    p0 = gf.construct_Green_function(g0)
    gf.update_potential(p0, w.Vcell, w.mats, w.offsets, layout="cells")
    gf.update_energy_parameter(p0, w.E, w.dVol)
    a, b = p0.export(), p1.export()
    for k in a:
        if k == "AtomMatrices":
            assert np.abs(a[k] - b[k]).max() <= 1e-15 * np.abs(a[k]).max()
        else:
            assert np.array_equal(a[k], b[k]), k
