"""Host mesh handling (CPU only): the .hmsh reader and writer, the wedge generator and
renumbering, the .hsln writer, and their error reporting."""
import os

import numpy as np
import pytest

import cfd_optimisations_b200 as H
import oracle as O


@pytest.mark.parametrize("nx,ny", [(161, 81), (41, 21), (7, 4)])
def test_generated_counts(nx, ny):
    # Ntri = 2(nx-1)(ny-1), Ng = 2(nx-1) + 2(ny-1), Nf = (nx-1)ny + nx(ny-1) + (nx-1)(ny-1)
    a = H.Mesh.wedge(nx, ny, seed=1).arrays()
    ntri, ng = 2 * (nx - 1) * (ny - 1), 2 * (nx - 1) + 2 * (ny - 1)
    assert a["Nc"] == ntri + ng
    assert a["Nf"] == (nx - 1) * ny + nx * (ny - 1) + (nx - 1) * (ny - 1)
    assert list(a["coltag"]) == [0, 1, 2, 3, 4]
    nbf = np.diff(a["coloff"])
    assert list(nbf[1:]) == [nx - 1, nx - 1, ny - 1, ny - 1]      # upper, lower, inlet, outlet
    assert a["pnames"] == ["upper", "lower", "inlet", "outlet"]


@pytest.mark.parametrize("numbering", [H.NUMBER_NATURAL, H.NUMBER_RANDOM, H.NUMBER_RCM, H.NUMBER_MORTON])
def test_face_conventions(numbering):
    """interface/Mesh.py:321-378: faces sorted by (min cell, max cell) inside each colour,
    interior faces CL < CR, ghost on the right of every boundary face, each ghost one face."""
    a = H.Mesh.wedge(41, 21, seed=6, numbering=numbering).arrays()
    fc = a["fc_con"].reshape(-1, 2)
    F_BC = a["coloff"][1]
    assert np.all(fc[:F_BC, 0] < fc[:F_BC, 1])
    for c in range(a["Ncol"]):
        blk = fc[a["coloff"][c]:a["coloff"][c + 1]]
        key = np.minimum(blk[:, 0], blk[:, 1]).astype(np.int64) * (1 << 32) + np.maximum(blk[:, 0], blk[:, 1])
        assert np.all(np.diff(key) > 0)
    ghosts = fc[F_BC:, 1]
    assert len(np.unique(ghosts)) == len(ghosts)
    deg = np.bincount(fc.ravel(), minlength=a["Nc"])
    assert np.all(deg[ghosts] == 1)
    assert np.all(np.diff(a["cn_off"])[ghosts] == 2)


def test_renumbering_preserves_the_mesh():
    """Every numbering describes the same cells: same multiset of (sorted) node lists."""
    sets = []
    for numbering in (H.NUMBER_NATURAL, H.NUMBER_RANDOM, H.NUMBER_RCM, H.NUMBER_MORTON):
        a = H.Mesh.wedge(21, 11, seed=9, numbering=numbering).arrays()
        cells = [tuple(sorted(a["cn_con"][a["cn_off"][c]:a["cn_off"][c + 1]])) for c in range(a["Nc"])]
        sets.append(sorted(cells))
    assert all(s == sets[0] for s in sets[1:])


def test_hmsh_round_trip(tmp_path):
    m = H.Mesh.wedge(41, 21, seed=5, numbering=H.NUMBER_RCM)
    p = str(tmp_path / "w.hmsh")
    m.write(p)
    a, b = m.arrays(), O.read_hmsh(p)
    for k in ("coltag", "coloff", "nodes", "fn_con", "fc_con", "cn_off", "cn_con", "cc_off", "cc_con"):
        assert np.array_equal(a[k], b[k]), k
    assert b["c_ctypes"] is not None and set(np.unique(b["c_ctypes"])) == {1, 2}
    c = H.Mesh(p).arrays()
    for k in ("coltag", "coloff", "nodes", "fn_con", "fc_con", "cn_off", "cn_con", "cf_off", "cf_con"):
        assert np.array_equal(a[k], c[k]), k


def test_reads_the_reference_mesh(golden):
    m = H.Mesh(os.path.join(golden, "wedge.hmsh"))
    a = m.arrays()
    assert (a["Nc"], a["Nf"], a["Nn"]) == (3740, 7120, 3621)
    assert a["pnames"] == ["upper", "lower", "inlet", "outlet"]
    # cell->face table of Mesh::compute_cf_con: faces of each cell in increasing order
    ref = O.read_hmsh(os.path.join(golden, "wedge.hmsh"))
    fc = ref["fc_con"].reshape(-1, 2)
    lists = [[] for _ in range(a["Nc"])]
    for f, (L, R) in enumerate(fc):
        lists[L].append(f)
        lists[R].append(f)
    assert np.array_equal(a["cf_con"], np.concatenate([np.array(x, dtype=np.int32) for x in lists]))


def test_cf_table_matches_reference_build(golden):
    if not O.RefSolver.available():
        pytest.skip("reference not compiled into oracle/_ref")
    import ctypes as ct
    path = os.path.join(golden, "wedge.hmsh")
    a = H.Mesh(path).arrays()
    off = np.zeros(a["Nc"] + 1, np.int32)
    con = np.zeros(2 * a["Nf"], np.int32)
    O.RefSolver.lib().hcfd_ref_mesh_cf(path.encode(), O._i(off), O._i(con))
    assert np.array_equal(off, a["cf_off"]) and np.array_equal(con, a["cf_con"])


def test_missing_and_truncated_files_are_errors(tmp_path, golden):
    with pytest.raises(H.HcfdError) as e:
        H.Mesh(str(tmp_path / "nope.hmsh"))
    assert e.value.code == -6
    with open(os.path.join(golden, "wedge.hmsh"), "rb") as fh:
        b = fh.read()
    for cut in (10, 200, len(b) // 2):
        p = tmp_path / f"cut{cut}.hmsh"
        p.write_bytes(b[:cut])
        with pytest.raises(H.HcfdError) as e:
            H.Mesh(str(p))
        assert e.value.code in (-6, -1)


def test_corrupted_connectivity_is_rejected(tmp_path, golden):
    a = O.read_hmsh(os.path.join(golden, "wedge.hmsh"))
    with open(os.path.join(golden, "wedge.hmsh"), "rb") as fh:
        b = bytearray(fh.read())
    # fc_con starts after header, names, coltag, coloff, nodes and fn_con
    off = 32 + 25 + 4 * 5 + 4 * 6 + 8 * 2 * a["Nn"] + 4 * 2 * a["Nf"]
    b[off:off + 4] = np.int32(10 ** 8).tobytes()      # a cell index far out of range
    p = tmp_path / "bad.hmsh"
    p.write_bytes(bytes(b))
    with pytest.raises(H.HcfdError) as e:
        H.Mesh(str(p))
    assert e.value.code == -1


@pytest.mark.parametrize("kw", [dict(nx=2, ny=5), dict(nx=5, ny=5, jitter=0.6), dict(nx=5, ny=5, theta_deg=80.0)])
def test_generator_rejects_bad_specs(kw):
    nx, ny = kw.pop("nx"), kw.pop("ny")
    with pytest.raises(H.HcfdError):
        H.Mesh.wedge(nx, ny, **kw)


def test_hsln_writer_round_trip(tmp_path):
    rng = np.random.default_rng(1)
    arrs = [rng.standard_normal(37) for _ in range(4)]
    p = str(tmp_path / "s_0.hsln")
    H.write_hsln(p, arrs)
    names, data = O.read_hsln(p)
    assert names == ["Density", "Velocity_X", "Velocity_Y", "Pressure"]
    assert np.array_equal(data, np.stack(arrs))


def test_hsln_header_matches_reference_writer(golden):
    """Same header bytes as the reference's Writer (src/Writer.cpp:28-34)."""
    with open(os.path.join(golden, "Base_0.hsln"), "rb") as fh:
        ref = fh.read()
    _, data = O.read_hsln(os.path.join(golden, "Base_0.hsln"))
    import tempfile
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "x.hsln")
        H.write_hsln(p, list(data))
        with open(p, "rb") as fh:
            mine = fh.read()
    assert mine == ref
