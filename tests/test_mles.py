"""The .mles reader (cgx_mles_read, include/cgx_mles.h) on the reference's
own mesher output, src/core/common/tests/assets/orifice.mles.

CPU only; skipped where the reference tree is absent.  The reference's test
of its reader (src/core/common/tests/testStripedMesh.cpp:13-22) pins the
counts.  The arrays are pinned by identities the file's geometry must satisfy
and by the zone totals Stitch writes into each boundary-zone header:
  * every cell closes: the outward area vectors of its faces and boundary
    faces sum to zero;
  * the divergence theorem gives vol_cv exactly for cells without boundary
    faces (all their faces are planar Voronoi polygons);
  * each face's area vector is the area vector of its node polygon;
  * each zone's area, area vector, area-weighted centroid and area_over_delta
    equal the sums over its faces.
"""
import os

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REFERENCE_ROOT = os.environ.get("REFERENCE_ROOT", "/root/reference")
ASSET = os.path.join(REFERENCE_ROOT, "src/core/common/tests/assets/orifice.mles")
V3_LES = os.path.join(REFERENCE_ROOT, "grids/result.lam_chan.les")

pytestmark = pytest.mark.skipif(not os.path.exists(ASSET), reason="reference tree not present")


@pytest.fixture(scope="module")
def mesh(built):
    from nextgen_b200.mles import MlesMesh
    return MlesMesh(ASSET)


def test_counts_match_the_reference_reader_test(mesh):
    # testStripedMesh.cpp:13-22 (nef_global == 0: no extended faces are stored)
    assert mesh.io_version == 5
    assert (mesh.nno, mesh.nbf, mesh.nfa, mesh.nfa_p, mesh.ncv, mesh.nno_p, mesh.nno_pb) == \
        (46348, 693, 5654, 0, 1056, 0, 42383)
    assert mesh.nfa_zone[26] == mesh.nfa and mesh.nfa_zone[:26].sum() == 0
    assert [z["name"] for z in mesh.bf_zones] == ["inlet", "outlet", "oriface-pipe", "wall", "oriface-wall-0",
                                                  "oriface-wall-1"]
    assert sum(z["nbf"] for z in mesh.bf_zones) == mesh.nbf and mesh.cv_zone_ncv == [mesh.ncv]
    for a in ("x_no", "cvofa", "noofa_i", "n_fa", "x_fa", "cvobf", "noobf_i", "n_bf", "x_bf", "area_bf",
              "area_over_delta_bf", "Gij_bf", "vol_cv", "r_vv", "x_vv", "x_cv"):
        assert getattr(mesh, a) is not None, a


def test_indices(mesh):
    assert (mesh.cvofa[:, 0] < mesh.cvofa[:, 1]).all() and mesh.cvofa.min() >= 0 and mesh.cvofa.max() < mesh.ncv
    assert mesh.cvobf.min() >= 0 and mesh.cvobf.max() < mesh.ncv
    assert mesh.noofa_v.min() >= 0 and mesh.noofa_v.max() < mesh.nno
    assert (np.diff(mesh.noofa_i) >= 3).all() and (np.diff(mesh.noobf_i) >= 3).all()


def _cell_sums(m):
    S = np.zeros((m.ncv, 3))
    A = np.zeros(m.ncv)
    np.add.at(S, m.cvofa[:, 0], m.n_fa)
    np.add.at(S, m.cvofa[:, 1], -m.n_fa)
    np.add.at(S, m.cvobf, m.n_bf)
    an, ab = np.linalg.norm(m.n_fa, axis=1), np.linalg.norm(m.n_bf, axis=1)
    np.add.at(A, m.cvofa[:, 0], an)
    np.add.at(A, m.cvofa[:, 1], an)
    np.add.at(A, m.cvobf, ab)
    return S, A


def test_cells_close(mesh):
    S, A = _cell_sums(mesh)
    assert (np.linalg.norm(S, axis=1) / A).max() < 1e-8


def test_divergence_volume_of_interior_cells(mesh):
    m = mesh
    V = np.zeros(m.ncv)
    xc = m.x_cv
    np.add.at(V, m.cvofa[:, 0], ((m.x_fa - xc[m.cvofa[:, 0]]) * m.n_fa).sum(1))
    np.add.at(V, m.cvofa[:, 1], -((m.x_fa - xc[m.cvofa[:, 1]]) * m.n_fa).sum(1))
    np.add.at(V, m.cvobf, ((m.x_bf - xc[m.cvobf]) * m.n_bf).sum(1))
    V /= 3.0
    interior = np.bincount(m.cvobf, minlength=m.ncv) == 0
    assert interior.sum() > 400
    assert (np.abs(V - m.vol_cv)[interior] / m.vol_cv[interior]).max() < 1e-12


def _poly_area(x_no, nodes, c):
    P = x_no[nodes]
    return 0.5 * np.cross(P - c, np.roll(P, -1, axis=0) - c).sum(0)


def test_area_vectors_are_the_node_polygons(mesh):
    m = mesh
    ef = np.array([np.linalg.norm(_poly_area(m.x_no, m.noofa_v[m.noofa_i[i]:m.noofa_i[i + 1]], m.x_fa[i]) - m.n_fa[i])
                   / np.linalg.norm(m.n_fa[i]) for i in range(m.nfa)])
    eb = np.array([np.linalg.norm(_poly_area(m.x_no, m.noobf_v[m.noobf_i[i]:m.noobf_i[i + 1]], m.x_bf[i]) - m.n_bf[i])
                   / np.linalg.norm(m.n_bf[i]) for i in range(m.nbf)])
    assert eb.max() < 1e-7
    # 9 of the 5654 faces (cut faces at the orifice) are not planar polygons
    assert (ef < 1e-6).sum() >= m.nfa - 10 and ef.max() < 0.5
    # the area of a boundary face is at least its projected area
    assert (m.area_bf >= np.linalg.norm(m.n_bf, axis=1) * (1 - 1e-12)).all()


def test_zone_totals(mesh):
    m = mesh
    for z in m.bf_zones:
        sl = slice(z["ibf_f"], z["ibf_f"] + z["nbf"])
        a = m.area_bf[sl].sum()
        assert abs(a - z["area"]) <= 1e-12 * z["area"]
        assert np.abs(m.n_bf[sl].sum(0) - z["n"]).max() <= 1e-12 * a
        x = (m.x_bf[sl] * m.area_bf[sl, None]).sum(0) / a
        assert np.abs(x - z["x"]).max() <= 1e-12 * (1.0 + np.abs(z["x"]).max())
        assert abs(m.area_over_delta_bf[sl].sum() - z["area_over_delta"]) <= 1e-12 * z["area_over_delta"]


def _records(data):
    """(offset, id, skip) of each record of a UGP record file: a 256-byte
    header per record, id at byte 52, skip (int64) at byte 56."""
    out, off = [], 8
    while off + 256 <= len(data):
        rid = int(np.frombuffer(data, np.int32, 1, off + 52)[0])
        skip = int(np.frombuffer(data, np.int64, 1, off + 56)[0])
        out.append((off, rid, skip))
        if rid == 51 or skip < 256:
            break
        off += skip
    return out


def test_errors(built, tmp_path):
    from nextgen_b200.mles import MlesError, MlesMesh
    with pytest.raises(MlesError) as e:
        MlesMesh(str(tmp_path / "restart.does.not.exist.mles"))
    assert e.value.code == -1
    txt = tmp_path / "not_a_mesh.mles"
    txt.write_bytes(b"RESTART tests/assets/orifice.mles\n" * 20)
    with pytest.raises(MlesError) as e:
        MlesMesh(str(txt))
    assert e.value.code == -2
    cut = tmp_path / "truncated.mles"
    cut.write_bytes(open(ASSET, "rb").read()[:1_500_000])
    with pytest.raises(MlesError) as e:
        MlesMesh(str(cut))
    assert e.value.code == -1
    # the same file with its first two words in the other byte order
    raw = bytearray(open(ASSET, "rb").read(1 << 16))
    for o in (0, 4):
        raw[o:o + 4] = raw[o:o + 4][::-1]
    swapped = tmp_path / "swapped.mles"
    swapped.write_bytes(bytes(raw))
    with pytest.raises(MlesError) as e:
        MlesMesh(str(swapped))
    assert e.value.code == -3 and "byte-swapped" in str(e.value)
    # a second counts record after the cell-face records were read at the
    # first one's sizes is refused
    data = open(ASSET, "rb").read()
    recs = _records(data)
    cnt = next(r for r in recs if r[1] == 10001)
    after = next(r for r in recs if r[1] == 2006)  # cvofa
    dup = data[:after[0] + after[2]] + data[cnt[0]:cnt[0] + cnt[2]] + data[after[0] + after[2]:]
    twice = tmp_path / "two_counts.mles"
    twice.write_bytes(dup)
    with pytest.raises(MlesError) as e:
        MlesMesh(str(twice))
    assert e.value.code == -2 and "second counts" in str(e.value)
    # a record whose count reaches past the end of the file is refused before
    # anything of that size is allocated: the x_no record cut after its header
    xno = next(r for r in recs if r[1] == 31)
    short = tmp_path / "short_x_no.mles"
    short.write_bytes(data[:xno[0] + 256 + 64])
    with pytest.raises(MlesError) as e:
        MlesMesh(str(short))
    assert e.value.code == -1 and "past the end" in str(e.value)
    if os.path.exists(V3_LES):
        with pytest.raises(MlesError) as e:
            MlesMesh(V3_LES)
        assert e.value.code == -3 and "io version 3" in str(e.value)
