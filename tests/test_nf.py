"""Neutral-file reader: round trips through the writer, and parity with the
reference's own FileIO::ReadNF (compiled oracle library) on the same files,
including files whose sections are out of the reader's scan order."""
import os
import tempfile

import numpy as np
import pytest

from gpufem_b200 import meshgen as mg
from gpufem_b200.nf import NfError, read_nf
from oracle.oracle import Reference

CASES = [
    (mg.Q4, (4, 3), 2),
    (mg.Q8, (3, 3), 3),
    (mg.BRICK8, (3, 2, 2), 2),
    (mg.BRICK20, (2, 2, 1), 3),
]


def _mesh(et, n, ngauss):
    m = mg.clamp_and_load(mg.structured(et, n, jitter=0.2, seed=7, ngauss=ngauss))
    return m


@pytest.mark.parametrize("et,n,ngauss", CASES)
def test_roundtrip(tmp_path, et, n, ngauss):
    m = _mesh(et, n, ngauss)
    path = str(tmp_path / "m.nf")
    mg.write_nf(m, path)
    r = read_nf(path)
    assert r.elem_type == et
    np.testing.assert_array_equal(r.coords, m.coords)
    np.testing.assert_array_equal(r.conn, m.conn)
    np.testing.assert_array_equal(r.supports, m.supports)
    f32 = m.f.astype(np.float32).astype(np.float64)   # loads are parsed as FP32
    np.testing.assert_array_equal(r.force_vector(), f32)
    mm = r.to_mesh(E=m.E0, nu=m.nu, ngauss=ngauss)
    assert mm.nelem == m.nelem and mm.ndof == m.ndof


@pytest.mark.skipif(not Reference.available("fp64"), reason="reference library not built")
@pytest.mark.parametrize("et,n,ngauss", CASES)
def test_matches_reference_reader(tmp_path, et, n, ngauss):
    m = _mesh(et, n, ngauss)
    path = str(tmp_path / "m.nf")
    mg.write_nf(m, path)
    r = read_nf(path)
    s = Reference("fp64").open(path, ngauss, m.E0, m.nu)
    try:
        np.testing.assert_array_equal(r.coords, s.coords())
        np.testing.assert_array_equal(r.conn, s.connect())
        np.testing.assert_array_equal(r.supports, s.supports())
        np.testing.assert_array_equal(r.force_vector(), s.force())
    finally:
        s.close()


_SCRAMBLED = """header line
%ELEMENT
2

%NODE.SUPPORT
2
1\t1\t1\t0\t0\t0\t0
4\t1\t0\t0\t0\t0\t0

%ELEMENT.Q4
2
1\t1\t1\t1\t1\t2\t5\t4
2\t1\t1\t1\t2\t3\t6\t5

%HEADER.ANALYSIS
'plane_stress'

%NODE.COORD
6
1\t0.0\t0.0\t0.0
2\t0.5\t0.0\t0.0
3\t1.0\t0.0\t0.0
4\t0.0\t1.0\t0.0
5\t0.5\t1.0\t0.0
6\t1.0\t1.0\t0.0

%LOAD.CASE.NODAL.FORCES
2
3\t0.1\t0.0\t0.0\t0.0\t0.0\t0.0
6\t0.1\t-0.3\t0.0\t0.0\t0.0\t0.0

%END
"""


def test_scrambled_sections_follow_reference_scan(tmp_path):
    """%NODE.SUPPORT before the element block is found only after the rewind at
    %END, exactly as FileIO::findParameter does."""
    path = str(tmp_path / "s.nf")
    with open(path, "w") as fh:
        fh.write(_SCRAMBLED)
    r = read_nf(path)
    assert r.elem_type == mg.Q4 and r.analysis == "'plane_stress'"
    np.testing.assert_array_equal(r.conn, [[1, 2, 5, 4], [2, 3, 6, 5]])
    np.testing.assert_array_equal(r.supports, [[1, 1, 1], [4, 1, 0]])
    f = r.force_vector()
    assert f[4] == np.float32(0.1) and f[10] == np.float32(0.1) and f[11] == np.float32(-0.3)
    if Reference.available("fp64"):
        s = Reference("fp64").open(path, 2, 210e3, 0.3)
        try:
            np.testing.assert_array_equal(r.coords, s.coords())
            np.testing.assert_array_equal(r.conn, s.connect())
            np.testing.assert_array_equal(r.supports, s.supports())
            np.testing.assert_array_equal(f, s.force())
        finally:
            s.close()


def test_rejects_bad_files(tmp_path):
    p = tmp_path / "x.txt"
    p.write_text("%ELEMENT.Q4\n0\n")
    with pytest.raises(NfError):
        read_nf(str(p))
    p = tmp_path / "y.nf"
    p.write_text("%ELEMENT.TRI3\n1\n1 1 1 1 1 2 3\n%END\n")
    with pytest.raises(NfError):
        read_nf(str(p))
    p = tmp_path / "z.nf"
    p.write_text("%ELEMENT.Q4\n1\n1 1 1 1 1 2 3 9\n%HEADER.ANALYSIS\n'plane_stress'\n"
                 "%NODE.COORD\n4\n1 0 0 0\n2 1 0 0\n3 1 1 0\n4 0 1 0\n%END\n")
    with pytest.raises(NfError):
        read_nf(str(p))


@pytest.mark.gpu
@pytest.mark.skipif(not Reference.available("fp64"), reason="reference library not built")
def test_nf_file_through_fem_facade_matches_reference(tmp_path):
    """A neutral file read here and by the reference gives the same displacements:
    FEM facade (read_nf -> gf_mesh_create -> assembly -> penalty -> CG) against the
    reference's ReadNF -> StiffAlgoCPU -> ApplyConstraint(PEN) -> CPU_CG."""
    from gpufem_b200 import _lib
    from gpufem_b200.fem import FEM
    m = _mesh(mg.Q8, (6, 5), 3)
    path = str(tmp_path / "q8.nf")
    mg.write_nf(m, path)
    fem = FEM()
    fem.Init()
    fem.GetFemData().InitFromFile(path, 3, 210e3, 0.3)
    fem.SetPrecision(_lib.GF_F64)
    fem.CalcStiffnessMat()
    fem.ApplyConstraint(FEM.PEN)
    u = fem.Solve(n_iterations=50000, epsilon=1e-10)
    s = Reference("fp64").open(path, 3, 210e3, 0.3)
    try:
        s.assemble()
        s.penalty()
        x, _ = s.cg(50000, 1e-10)
    finally:
        s.close()
    assert np.linalg.norm(u - x) <= 1e-6 * np.linalg.norm(x)


def test_write_xyz_vector_format(tmp_path):
    from gpufem_b200.nf import write_xyz_vector
    p = str(tmp_path / "out.txt")
    write_xyz_vector(p, np.array([1.0, -2.5, 0.125, 10.0, 0.0, -0.004, 7.0]), append=False)
    text = open(p).read()
    assert text == ("\nDisplacement Vector Dump:\n Node+===x===+===y===+===z===+\n"
                    "  1 -    1.00   -2.50    0.12\n"
                    "  2 -   10.00    0.00   -0.00\n")
