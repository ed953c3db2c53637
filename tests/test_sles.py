""".sles result files (cgx_sles_write / cgx_sles_read, the record layout of
StaticSolver::writeData and CtiData::writeData,
src/core/common/StaticSolver.cpp:7560-7640, CtiRegister.cpp:412-610) and the
compact orifice fixture, on CPU."""
import os

import numpy as np
import pytest

from nextgen_b200.mles import CompactMesh, MlesError, read_sles, write_sles

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURE = os.path.join(HERE, "golden", "orifice_compact.npz")
REFERENCE_ROOT = os.environ.get("REFERENCE_ROOT", "/root/reference")
ASSET = os.path.join(REFERENCE_ROOT, "src/core/common/tests/assets/orifice.mles")


def _records(data):
    out, off = [], 8
    while off + 256 <= len(data):
        name = data[off:off + 52].split(b"\0")[0].decode()
        rid = int(np.frombuffer(data, np.int32, 1, off + 52)[0])
        skip = int(np.frombuffer(data, np.int64, 1, off + 56)[0])
        out.append((name, rid, skip, off))
        if rid == 51:
            break
        off += skip
    return out


def test_round_trip_and_layout(built, tmp_path):
    rng = np.random.default_rng(2)
    n = 1000
    rho, u, rhoE = rng.uniform(0.5, 2, n), rng.normal(size=(n, 3)), rng.uniform(1, 5, n)
    p = tmp_path / "result.00000042.sles"
    write_sles(p, rho, u, rhoE, step=42, time=1.25, params="GAMMA 1.4\n")
    r2, u2, e2, st, t = read_sles(p, n)
    assert np.array_equal(r2, rho) and np.array_equal(u2, u) and np.array_equal(e2, rhoE)
    assert (st, t) == (42, 1.25)
    data = p.read_bytes()
    assert tuple(np.frombuffer(data, np.int32, 2)) == (123581322, 5)
    recs = _records(data)
    assert [(r[0], r[1]) for r in recs] == [("UGP_IO_HASHIDS", 94), ("UGP_IO_PARAMS", 91), ("rho", 42),
                                            ("rhoE", 42), ("step", 11), ("time", 12), ("u", 43), ("EOF", 51)]
    name, _, skip, off = recs[6]
    assert skip == 256 + 24 * n
    assert np.array_equal(np.frombuffer(data, np.float64, 3 * n, off + 256).reshape(n, 3), u)
    assert recs[-1][3] + 256 == len(data)
    assert not os.path.exists(str(p) + ".tmp")


def test_errors(built, tmp_path):
    n = 10
    p = tmp_path / "a.sles"
    write_sles(p, np.ones(n), np.zeros((n, 3)), np.ones(n))
    with pytest.raises(MlesError) as e:
        read_sles(p, n + 1)  # another mesh
    assert e.value.code == -2
    data = p.read_bytes()
    (tmp_path / "cut.sles").write_bytes(data[: len(data) // 2])
    with pytest.raises(MlesError) as e:
        read_sles(tmp_path / "cut.sles", n)
    assert e.value.code == -1
    (tmp_path / "mesh.sles").write_bytes(np.array([123581321, 5], np.int32).tobytes() + data[8:])
    with pytest.raises(MlesError) as e:
        read_sles(tmp_path / "mesh.sles", n)
    assert e.value.code == -2


def test_orifice_fixture(built):
    c = CompactMesh.load(FIXTURE)
    assert (c.ncv, c.nfa, c.nbf) == (1056, 5654, 693)
    assert c.zone_names == ["inlet", "outlet", "oriface-pipe", "wall", "oriface-wall-0", "oriface-wall-1"]
    assert (c.cvofa[:, 0] < c.cvofa[:, 1]).all() and (np.diff(c.cvofa[:, 0]) >= 0).all()
    S = np.zeros((c.ncv, 3))
    np.add.at(S, c.cvofa[:, 0], c.n_fa)
    np.add.at(S, c.cvofa[:, 1], -c.n_fa)
    np.add.at(S, c.cvobf, c.n_bf)
    A = np.zeros(c.ncv)
    a = np.linalg.norm(c.n_fa, axis=1)
    np.add.at(A, c.cvofa[:, 0], a)
    np.add.at(A, c.cvofa[:, 1], a)
    np.add.at(A, c.cvobf, c.area_bf)
    assert (np.linalg.norm(S, axis=1) / A).max() < 1e-8
    if os.path.exists(ASSET):
        from nextgen_b200.mles import MlesMesh
        d = CompactMesh.from_mles(MlesMesh(ASSET))
        for k in CompactMesh.FIELDS:
            assert np.array_equal(getattr(d, k), getattr(c, k)), k
