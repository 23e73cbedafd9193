"""OFELI's .m mesh files on the host (no GPU): ofg_mesh_file_read /
ofg_mesh_file_write against the reference's own Mesh::get / Mesh::put
(golden outputs in tests/golden/meshio.npz, and every demo mesh of the
reference when its sources and harness are present) and against the oracle
restatement (oracle/mesh_oracle.py).

Bars: every array bit-exact (coordinates are OFELI's float-rounded values),
put output byte-identical, the same files rejected."""
import glob
import os
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import GOLDEN, REFERENCE, load_golden
from ofeli_b200 import ofeli as F
from ofeli_b200 import problems
from oracle import mesh_oracle as MO
from oracle import oracle as O

FILES = ("ring", "codes", "tet")
REF_DEMOS = sorted(glob.glob(os.path.join(REFERENCE, "demos/**/*.m"), recursive=True)
                   + glob.glob(os.path.join(REFERENCE, "util/cmesh/disk.m")))


@pytest.fixture(scope="module")
def golden():
    return load_golden("meshio")


def arrays_of(path):
    mf = F.MeshFile(path)
    return mf, mf.arrays()


def assert_same(a, g, key):
    assert np.array_equal(a["coords"].ravel(), g[key + "_coords"])
    assert np.array_equal(a["node_code"].ravel(), g[key + "_node_code"])
    assert np.array_equal(a["elem"].ravel(), g[key + "_elem"])
    assert np.array_equal(a["elem_code"].ravel(), g[key + "_elem_code"])
    assert np.array_equal(a["sides"].ravel(), g[key + "_side"])
    assert np.array_equal(a["side_code"].ravel(), g[key + "_side_code"])


@pytest.mark.parametrize("key", FILES)
def test_read_matches_reference(golden, key):
    g, info = golden
    mf, a = arrays_of(os.path.join(GOLDEN, "meshio_%s.m" % key))
    meta = info["files"][key]
    assert (mf.dim, mf.nb_dof, mf.nn, mf.ne, mf.ns) == (meta["dim"], meta["nb_dof"], meta["nodes"],
                                                        meta["elements"], meta["sides"])
    assert (mf.el_shape, mf.el_nodes) == (meta["el_shape"], meta["el_nodes"])
    if mf.ns:
        assert (mf.sd_shape, mf.sd_nodes) == (meta["sd_shape"], meta["sd_nodes"])
    assert_same(a, g, key)


@pytest.mark.parametrize("key", FILES)
def test_put_matches_reference(golden, key, tmp_path):
    g, _ = golden
    mf = F.MeshFile(os.path.join(GOLDEN, "meshio_%s.m" % key))
    out = tmp_path / "put.m"
    mf.put(out)
    assert out.read_bytes() == g[key + "_put"].tobytes()


@pytest.mark.parametrize("key", FILES)
def test_oracle_pinned(golden, key):
    g, _ = golden
    m = MO.read(os.path.join(GOLDEN, "meshio_%s.m" % key))
    assert_same(dict(m, sides=m["sides"]), g, key)
    assert MO.put(m) == g[key + "_put"].tobytes()


def test_codes_quirks(golden):
    """DOFCode gives |digits| for a negative mark; put writes the codes back
    as one number per node (-12 -> 12) and an empty Material block when no
    element has code 1."""
    _, a = arrays_of(os.path.join(GOLDEN, "meshio_codes.m"))
    assert a["node_code"].tolist()[:4] == [[1, 1], [1, 2], [0, 3], [0, 1]]
    assert a["node_code"].tolist()[5:] == [[12, 0], [9, 9]]
    assert a["side_code"].tolist() == [[2, 1], [1, 0], [0, 0], [0, 3]]
    assert a["coords"][5, 0] == float(np.float32(0.1)) != 0.1
    assert b"   <Material>\n   </Material>\n" in golden[0]["codes_put"].tobytes()


@pytest.mark.skipif(not (REF_DEMOS and O.have_reference("o2") and
                         os.path.isdir(os.path.join(REFERENCE, "demos"))),
                    reason="needs the reference sources and oracle/_ref")
@pytest.mark.parametrize("path", REF_DEMOS, ids=lambda p: os.path.relpath(p, REFERENCE))
def test_reference_demo_meshes(path):
    """Every mesh file the reference ships: Mesh::get's arrays and Mesh::put's
    bytes (harness run here) against the library and the oracle."""
    if "<Mesh" not in open(path, errors="replace").read():
        pytest.skip("not a mesh file")
    tmp = tempfile.mkdtemp(prefix="mget_")
    info, out = O.run_reference(["mget", path], {}, keep=tmp)
    put = open(os.path.join(tmp, "out", "put.m"), "rb").read()
    g = {"x_coords": out["coords"], "x_node_code": out["node_code"], "x_elem": out["elem"] - 1,
         "x_elem_code": out["elem_code"], "x_side": out["side"] - 1,
         "x_side_code": out["side_code"]}
    mf, a = arrays_of(path)
    assert_same(a, g, "x")
    p = os.path.join(tmp, "ours.m")
    mf.put(p)
    assert open(p, "rb").read() == put
    m = MO.read(path)
    assert_same(m, g, "x")
    assert MO.put(m) == put


TOKENS = ["0.1", "1e-1", "-2.5E+3", "3.14159265358979", "+1.5", ".5", "5.", "1e", "-0", "0",
          "0.0e0", "0x1p-3", "-0x1.8p1", "inf", "-Infinity", "nan", "1.17549435e-38",
          "3.40282346e38", "16777217", "0.30000001192092896", "7.0000004", "1.00000005e-01",
          "123456789012345678901234567890", "1e-30"]


def nodes_file(path, tokens):
    body = "".join("  %s 0.0 %d\n" % (t, i % 3) for i, t in enumerate(tokens))
    with open(path, "w") as fh:
        fh.write('<?xml version="1.0"?>\n<OFELI_File>\n<Mesh dim="2" nb_dof="1">\n<Nodes>\n'
                 + body + "</Nodes>\n</Mesh>\n</OFELI_File>\n")


def test_coordinates_round_like_stof(tmp_path):
    """Decimal, signed, hexadecimal, infinite and NaN forms convert to the
    value std::stof gives (strtof, here through the oracle)."""
    rng = np.random.default_rng(3)
    rand = ["%.*e" % (int(d), v) for d, v in zip(rng.integers(0, 17, 400),
                                                   rng.standard_normal(400) * 10.0 **
                                                   rng.integers(-30, 30, 400))]
    p = tmp_path / "nodes.m"
    nodes_file(p, TOKENS + rand)
    _, a = arrays_of(p)
    m = MO.read(p)
    assert np.array_equal(a["coords"].view(np.int64), m["coords"].view(np.int64))
    for tok, v in zip(TOKENS + rand, a["coords"][:, 0]):
        assert np.float32(v) == v or np.isnan(v)
        assert (np.isnan(v) and np.isnan(MO.stof(tok))) or v == MO.stof(tok)


@pytest.mark.parametrize("tok", ["1e39", "-1e39", "1e-46", "9.99999944e-39", "abc", "-", "e5"])
def test_coordinates_stof_rejects(tmp_path, tok):
    p = tmp_path / "bad.m"
    nodes_file(p, ["1.0", tok])
    with pytest.raises(F.OFELIException):
        F.MeshFile(p)
    with pytest.raises(MO.MeshFileError):
        MO.read(p)


BAD = {
    "single_quotes": "<OFELI_File><Mesh dim='2'></Mesh></OFELI_File>",
    "space_before_eq": '<OFELI_File><Mesh dim ="2"></Mesh></OFELI_File>',
    "unclosed_root": '<OFELI_File><Mesh dim="2"></Mesh>',
    "mismatch": '<OFELI_File><Mesh dim="2"></Nodes></OFELI_File>',
    "gt_in_text": '<OFELI_File>a > b</OFELI_File>',
    "text_outside": 'x<OFELI_File></OFELI_File>',
    "space_in_close": '<OFELI_File></OFELI_File >',
    "pi_inside": '<OFELI_File><?x?></OFELI_File>',
    "int_overflow": '<OFELI_File><Mesh dim="2"><Nodes>0 0 99999999999</Nodes></Mesh></OFELI_File>',
    "bad_int": '<OFELI_File><Mesh dim="2"><Nodes>0 0 x</Nodes></Mesh></OFELI_File>',
}
# refused here where OFELI's reading is undefined (records cut short, labels
# outside the node list, fixed arrays overrun, unset shapes) or not mirrored
# (a block split by a comment restarts OFELI's labels; entity references)
REFUSED_HERE = {
    "cut_record": '<OFELI_File><Mesh dim="2"><Nodes>0 0 1 1</Nodes></Mesh></OFELI_File>',
    "label_zero": '<OFELI_File><Mesh dim="2"><Nodes>0 0 1 1 0 1 0 1 1</Nodes>'
                  '<Elements shape="triangle" nodes="3">0 1 2 1</Elements></Mesh></OFELI_File>',
    "label_past_end": '<OFELI_File><Mesh dim="2"><Nodes>0 0 1 1 0 1 0 1 1</Nodes>'
                      '<Elements shape="triangle" nodes="3">1 2 4 1</Elements></Mesh></OFELI_File>',
    "no_nodes_attr": '<OFELI_File><Mesh dim="2"><Nodes>0 0 1 1 0 1 0 1 1</Nodes>'
                     '<Elements shape="triangle">1 2 3 1</Elements></Mesh></OFELI_File>',
    "bad_side_shape": '<OFELI_File><Mesh dim="2"><Nodes>0 0 1 1 0 1</Nodes>'
                      '<Sides shape="curve" nodes="2">1 2 1</Sides></Mesh></OFELI_File>',
    "split_block": '<OFELI_File><Mesh dim="2"><Nodes>0 0 1<!-- c -->1 0 1</Nodes></Mesh>'
                   '</OFELI_File>',
    "dim_4": '<OFELI_File><Mesh dim="4"><Nodes>0 0 0 0 1</Nodes></Mesh></OFELI_File>',
    "nb_dof_7": '<OFELI_File><Mesh dim="2" nb_dof="7"><Nodes>0 0 1</Nodes></Mesh></OFELI_File>',
    "entity_in_data": '<OFELI_File><Mesh dim="2"><Nodes>0 0 &#49;</Nodes></Mesh></OFELI_File>',
}


@pytest.mark.parametrize("name", sorted(BAD) + sorted(REFUSED_HERE))
def test_rejects(tmp_path, name):
    p = tmp_path / (name + ".m")
    p.write_text(BAD.get(name) or REFUSED_HERE[name])
    with pytest.raises(F.OFELIException):
        F.MeshFile(p)
    with pytest.raises(MO.MeshFileError):
        MO.read(p)


@pytest.mark.skipif(not O.have_reference("o2"), reason="needs oracle/_ref")
@pytest.mark.parametrize("name", sorted(BAD))
def test_reference_rejects_too(tmp_path, name):
    """The malformed files OFELI itself refuses (an exception, exit status 3);
    files whose reading is undefined in OFELI are not run there."""
    p = tmp_path / (name + ".m")
    p.write_text(BAD[name])
    with pytest.raises(subprocess.CalledProcessError) as e:
        O.run_reference(["mget", str(p)], {}, timeout=60)
    assert e.value.returncode == 3


def test_threads_give_identical_results(tmp_path):
    """A file of a few MB cut into different numbers of chunks."""
    xy, elem, code, sides, smark = problems.ring_mesh(120, 300, seed=4)
    mf = F.MeshFile.create(2, xy, code, elem, np.ones(elem.shape[0], np.int32), F.TRIANGLE,
                           sides=sides, side_code=smark)
    p = tmp_path / "big.m"
    mf.put(p)
    assert os.path.getsize(p) > 3 << 20
    ref = None
    try:
        for t in (1, 2, 3, 7, 16, 0):
            F.MeshFile.set_threads(t)
            a = F.MeshFile(p).arrays()
            q = tmp_path / ("put%d.m" % t)
            F.MeshFile(p).put(q)
            if ref is None:
                ref, ref_put = a, q.read_bytes()
            for k in ref:
                assert np.array_equal(a[k], ref[k]), (t, k)
            assert q.read_bytes() == ref_put
    finally:
        F.MeshFile.set_threads(0)
    assert np.array_equal(ref["elem"], elem) and np.array_equal(ref["sides"], sides)
    m = MO.read(p)
    assert np.array_equal(ref["coords"], m["coords"]) and MO.put(m) == ref_put


def test_create_put_read_roundtrip(tmp_path):
    """Arrays -> put -> read: coordinates come back as OFELI's stof of the
    8-digit text, codes and topology unchanged."""
    xy, elem, code, sides, smark = problems.ring_mesh(5, 16, seed=6)
    ecode = (np.arange(elem.shape[0]) % 3 + 1).astype(np.int32)
    mf = F.MeshFile.create(2, xy, code, elem, ecode, F.TRIANGLE, sides=sides, side_code=smark)
    p = tmp_path / "r.m"
    mf.put(p)
    a = F.MeshFile(p).arrays()
    assert np.array_equal(a["elem"], elem) and np.array_equal(a["elem_code"], ecode)
    assert np.array_equal(a["node_code"].ravel(), code)
    assert np.array_equal(a["side_code"].ravel(), smark)
    expect = np.array([[MO.stof("%.8e" % v) for v in row] for row in xy])
    assert np.array_equal(a["coords"], expect)
    # the float-rounded coordinates print differently from the originals
    q = tmp_path / "r2.m"
    F.MeshFile(p).put(q)
    assert MO.put(MO.read(p)) == q.read_bytes() != p.read_bytes()
