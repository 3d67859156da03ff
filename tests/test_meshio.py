"""gmsh import and .vtu export on the CPU: a small mixed triangle/quadrangle mesh written as gmsh
4.1 ASCII, imported to .hmsh, loaded by the library's checked reader and stepped by the oracle;
solutions exported to .vtu and read back."""
import base64
import os
import struct
import xml.etree.ElementTree as ET

import numpy as np
import pytest

import cfd_optimisations_b200 as H
from cfd_optimisations_b200 import meshio
import oracle as O


def _msh_text(xy, curves, quads, tris, untagged_curve=None):
    """gmsh 4.1 ASCII text: nodes 1..len(xy); curve c (1-based) of `curves` = (physical tag,
    name, line elements) as an entity with that tag (none for `untagged_curve`); quadrangles
    and triangles (node tags) in one surface with physical tag 9 "domain", named last."""
    n = len(curves)
    L = ["$MeshFormat", "4.1 0 8", "$EndMeshFormat", "$PhysicalNames", str(n + 1)]
    for tag, name, _ in curves:
        L.append(f'1 {tag} "{name}"')
    L.append('2 9 "domain"')
    L += ["$EndPhysicalNames", "$Entities", f"4 {n} 1 0"]
    for p in range(1, 5):
        L.append(f"{p} 0 0 0 0")
    for c, (tag, _, _) in enumerate(curves, 1):
        ph = "0" if c == untagged_curve else f"1 {tag}"
        L.append(f"{c} 0 0 0 2 1 0 {ph} 2 {c} {-(c % 4 + 1)}")
    L.append(f"1 0 0 0 2 1 0 1 9 {n} " + " ".join(str(c) for c in range(1, n + 1)))
    L += ["$EndEntities", "$Nodes", f"1 {len(xy)} 1 {len(xy)}", f"2 1 0 {len(xy)}"]
    L += [str(t) for t in range(1, len(xy) + 1)]
    L += [f"{float(x)!r} {float(y)!r} 0" for x, y in xy]
    L.append("$EndNodes")
    blocks, tag = [], 1
    for c, (_, _, lines) in enumerate(curves, 1):
        blocks.append((1, c, 1, lines))
    blocks += [b for b in ((2, 1, 3, quads), (2, 1, 2, tris)) if len(b[3])]
    nel = sum(len(b[3]) for b in blocks)
    L += ["$Elements", f"{len(blocks)} {nel} 1 {nel}"]
    for d, e, t, els in blocks:
        L.append(f"{d} {e} {t} {len(els)}")
        for el in els:
            L.append(" ".join(str(x) for x in (tag,) + tuple(el)))
            tag += 1
    L.append("$EndElements")
    return "\n".join(L) + "\n"


def write_msh(path, nx=9, ny=5, tags=(1, 2, 3, 4), untagged_curve=None, with_quads=True):
    """Rectangle [0,2]x[0,1]: quadrangles in the left half (none without `with_quads`), triangles in
    the right half; curves bottom, right, top, left with physical tags `tags`, the surface with
    tag 9."""
    xs, ys = np.linspace(0, 2, nx), np.linspace(0, 1, ny)
    nid = lambda i, j: 1 + j * nx + i
    xy = [(xs[i], ys[j]) for j in range(ny) for i in range(nx)]
    quads, tris = [], []
    for j in range(ny - 1):
        for i in range(nx - 1):
            a, b, c, d = nid(i, j), nid(i + 1, j), nid(i + 1, j + 1), nid(i, j + 1)
            if with_quads and i < (nx - 1) // 2:
                quads.append((a, b, c, d))
            else:
                tris += [(a, b, c), (a, c, d)]
    sides = {1: [(nid(i, 0), nid(i + 1, 0)) for i in range(nx - 1)],
             2: [(nid(nx - 1, j), nid(nx - 1, j + 1)) for j in range(ny - 1)],
             3: [(nid(i + 1, ny - 1), nid(i, ny - 1)) for i in range(nx - 1)],
             4: [(nid(0, j + 1), nid(0, j)) for j in range(ny - 1)]}
    names = {1: "lower", 2: "outlet", 3: "upper", 4: "inlet"}
    curves = [(tags[c - 1], names[c], sides[c]) for c in (1, 2, 3, 4)]
    with open(path, "w") as fh:
        fh.write(_msh_text(xy, curves, quads, tris, untagged_curve))
    return dict(nquads=len(quads), ntris=len(tris), nlines=sum(len(v) for v in sides.values()))


def write_msh_of_mesh(path, m):
    """A library mesh (Mesh.arrays()) as gmsh: its real cells as surface elements, each
    boundary colour k (1-based) as a curve with physical tag k and the colour's name whose line
    elements are that colour's ghost cells (two nodes each)."""
    xy = m["nodes"].reshape(-1, 2)
    cn_off, cn_con = m["cn_off"], m["cn_con"]
    fc, coloff = m["fc_con"].reshape(-1, 2), m["coloff"]
    cell = lambda c: tuple(int(n) + 1 for n in cn_con[cn_off[c]:cn_off[c + 1]])
    ghosts = set(int(g) for g in fc[coloff[1]:, 1])
    real = [c for c in range(m["Nc"]) if c not in ghosts]
    curves = [(k, m["pnames"][k - 1], [cell(fc[f, 1]) for f in range(coloff[k], coloff[k + 1])])
              for k in range(1, m["Ncol"])]
    quads = [cell(c) for c in real if cn_off[c + 1] - cn_off[c] == 4]
    tris = [cell(c) for c in real if cn_off[c + 1] - cn_off[c] == 3]
    with open(path, "w") as fh:
        fh.write(_msh_text([tuple(p) for p in xy], curves, quads, tris))


def test_import_builds_a_valid_mesh(tmp_path):
    info = write_msh(tmp_path / "r.msh", tags=(3, 5, 7, 8))
    m = meshio.import_msh(str(tmp_path / "r.msh"), str(tmp_path / "r.hmsh"))
    nreal = info["nquads"] + info["ntris"]
    assert m["Nc"] == nreal + info["nlines"]
    mesh = H.Mesh(str(tmp_path / "r.hmsh"))          # the library's checked reader accepts it
    a = mesh.arrays()
    assert a["Nc"] == m["Nc"] and a["Nf"] == m["Nf"] and a["Ncol"] == 5 and a["NBCcol"] == 4
    assert a["pnames"] == ["lower", "outlet", "upper", "inlet"]            # tags 3 < 5 < 7 < 8
    fc = a["fc_con"].reshape(-1, 2)
    ctypes = m["c_ctypes"]
    F_BC = a["coloff"][1]
    assert np.all(ctypes[fc[F_BC:, 1]] == 1) and np.all(ctypes[fc[F_BC:, 0]] != 1)   # ghosts on the right
    assert np.all(ctypes[fc[:F_BC].ravel()] != 1) and np.all(fc[:F_BC, 0] < fc[:F_BC, 1])
    assert np.all(np.diff(a["coloff"]) == [m["Nf"] - info["nlines"], 8, 4, 8, 4])
    # every real cell has as many faces as sides
    deg = np.bincount(fc.ravel(), minlength=m["Nc"])
    assert np.all(deg[ctypes == 3] == 4) and np.all(deg[ctypes == 2] == 3) and np.all(deg[ctypes == 1] == 1)


def test_imported_mesh_keeps_a_uniform_flow_uniform(tmp_path):
    """Green-Gauss of a constant and the sum of a constant flux vanish on closed cells: the
    oracle stepping a freestream on the imported mesh must leave it unchanged."""
    write_msh(tmp_path / "r.msh")
    meshio.import_msh(str(tmp_path / "r.msh"), str(tmp_path / "r.hmsh"))
    mesh = H.Mesh(str(tmp_path / "r.hmsh"))
    o = O.Oracle(mesh.arrays())
    q = [1.4, 2.5, 0.3, 1.0]
    o.gather_bcs([O.SYMMETRY, O.SUPINLET, O.SUPINLET, O.SUPINLET, O.SUPINLET], [q] * 4)
    o.initialise(q)
    U0 = o.U()
    for _ in range(5):
        o.step(O.FIXED_DT, 1e-3)
    assert np.max(np.abs(o.U() - U0)) <= 1e-12 * np.max(np.abs(U0))


def test_import_errors(tmp_path):
    write_msh(tmp_path / "u.msh", untagged_curve=2)
    with pytest.raises(meshio.MshError, match="no physical tag"):
        meshio.import_msh(str(tmp_path / "u.msh"), str(tmp_path / "u.hmsh"))
    (tmp_path / "v.msh").write_text("$MeshFormat\n2.2 0 8\n$EndMeshFormat\n")
    with pytest.raises(meshio.MshError, match="4.x ASCII"):
        meshio.read_msh(str(tmp_path / "v.msh"))


def decode(arr):
    raw = base64.b64decode(arr.text)
    n = struct.unpack_from("<I", raw)[0]
    dt = {"Float64": np.float64, "Int64": np.int64, "UInt8": np.uint8}[arr.get("type")]
    return np.frombuffer(raw[4:4 + n], dtype=dt)


def test_export_vtu_round_trip(tmp_path):
    write_msh(tmp_path / "r.msh")
    m = meshio.import_msh(str(tmp_path / "r.msh"), str(tmp_path / "r.hmsh"))
    rng = np.random.default_rng(1)
    data = rng.normal(size=(4, m["Nc"]))
    names = ["Density", "Velocity_X", "Velocity_Y", "Pressure"]
    H.write_hsln(str(tmp_path / "s_3.hsln"), list(data), names)
    meshio.main(["export", str(tmp_path / "r.hmsh"), str(tmp_path / "s_3.hsln"), str(tmp_path / "s.vtu")])
    piece = ET.parse(tmp_path / "s.vtu").getroot().find("UnstructuredGrid/Piece")
    assert int(piece.get("NumberOfCells")) == m["Nc"] and int(piece.get("NumberOfPoints")) == m["Nn"]
    cells = {a.get("Name"): decode(a) for a in piece.find("Cells")}
    assert np.array_equal(cells["connectivity"], m["cn_con"]) and np.array_equal(cells["offsets"], m["cn_off"][1:])
    assert set(np.unique(cells["types"])) == {3, 5, 9}
    cd = {a.get("Name"): decode(a) for a in piece.find("CellData")}
    assert np.array_equal(cd["Density"], data[0]) and np.array_equal(cd["Pressure"], data[3])
    vel = cd["Velocity"].reshape(-1, 3)
    assert np.array_equal(vel[:, 0], data[1]) and np.array_equal(vel[:, 1], data[2]) and not vel[:, 2].any()
    out = meshio.batch_export(str(tmp_path / "r.hmsh"), str(tmp_path / "s_%d.hsln"), str(tmp_path / "o_%d.vtu"))
    assert out == [str(tmp_path / "o_3.vtu")]
    assert meshio.check_cell(str(tmp_path / "r.hmsh"), 0)["cell"] == 0


@pytest.mark.skipif(not O.RefSolver.available(), reason="reference not compiled into oracle/_ref")
def test_oracle_matches_reference_on_an_imported_mixed_mesh(tmp_path):
    """The reference's Base solver (compiled unchanged) reads the imported quadrangle/triangle
    mesh with its own reader and steps it; the oracle stays bit-identical to it, so the GPU's
    parity against the oracle on this mesh is parity against the reference."""
    write_msh(tmp_path / "r.msh", nx=41, ny=21)
    meshio.import_msh(str(tmp_path / "r.msh"), str(tmp_path / "r.hmsh"))
    path = str(tmp_path / "r.hmsh")
    bcmap = [O.SYMMETRY, O.SYMMETRY, O.SUPOUTLET, O.SYMMETRY, O.SUPINLET]
    q = np.array([1.4, 2.2, 0.35, 1.0])
    qbc = np.tile(q, (4, 1))
    o = O.Oracle(O.read_hmsh(path))
    o.gather_bcs(bcmap, qbc)
    o.initialise(q)
    U0 = o.U()
    dts = [o.step(O.GLOBAL_CFL, 0.5)[0] for _ in range(50)]
    r = O.RefSolver(path, np.array(bcmap), qbc, q)
    r.steps(50, np.array(dts))
    assert np.max(np.abs(o.U() - U0)) > 1e-2          # the walls have turned the flow
    assert np.array_equal(o.U(), r.U())


def _canonical(m):
    """A mesh up to its numbering: cells as (node count, node coordinates); faces as (node coordinates
    of the face, its two cells, colour name or 'interior').  A boundary face's cells are ordered
    (interior cell, ghost); an interior face's are unordered, since which of its cells is on the
    left follows the numbering (the lower number, in both importers)."""
    xy = m["nodes"].reshape(-1, m["dim"])
    node = lambda n: (float(xy[n, 0]), float(xy[n, 1]))
    cells = [(int(m["cn_off"][c + 1] - m["cn_off"][c]), frozenset(node(n) for n in m["cn_con"][m["cn_off"][c]:m["cn_off"][c + 1]]))
             for c in range(m["Nc"])]
    names = ["interior"] + list(m["pnames"])
    fn, fc, coloff = m["fn_con"].reshape(-1, 2), m["fc_con"].reshape(-1, 2), m["coloff"]
    faces = set()
    for col in range(m["Ncol"]):
        for f in range(coloff[col], coloff[col + 1]):
            pair = (cells[fc[f, 0]], cells[fc[f, 1]]) if col else frozenset((cells[fc[f, 0]], cells[fc[f, 1]]))
            faces.add((frozenset(node(n) for n in fn[f]), pair, names[col]))
    return sorted(cells, key=repr), faces


def test_import_matches_the_reference_importer_up_to_numbering(tmp_path, golden):
    """The reference's own importer (interface/Mesh.py, output committed by
    tests/golden/make_import_golden.py) and meshio.import_msh, on the same triangle-only gmsh
    file, give the same mesh: the same cells, the same faces with the same left/right cells
    (the ghost on the right) and colours, the same colour names and counts.  The numbering
    differs: the reference orders all cells, ghosts included, by one reverse Cuthill-McKee pass."""
    write_msh(tmp_path / "t.msh", nx=9, ny=5, with_quads=False)
    meshio.import_msh(str(tmp_path / "t.msh"), str(tmp_path / "t.hmsh"))
    ours = O.read_hmsh(str(tmp_path / "t.hmsh"))
    ref = O.read_hmsh(os.path.join(golden, "ref_import_tri.hmsh"))
    for k in ("dim", "Nn", "Nc", "Nf", "Ncol", "NBCcol", "pnames"):
        assert ours[k] == ref[k], k
    assert np.array_equal(np.diff(ours["coloff"]), np.diff(ref["coloff"]))
    cells_a, faces_a = _canonical(ours)
    cells_b, faces_b = _canonical(ref)
    assert cells_a == cells_b
    assert faces_a == faces_b and len(faces_a) == ours["Nf"]


def test_generated_wedge_matches_the_reference_importer_up_to_numbering(golden):
    """The wedge generator's mesh (13 x 7 nodes, seed 3, random numbering), written as gmsh and
    imported by the reference's own importer (output committed by
    tests/golden/make_import_golden.py), is the same mesh: the generator builds its cells, faces,
    boundary orientation and colours as the reference's mesh pipeline does."""
    m = H.Mesh.wedge(13, 7, seed=3, numbering=H.NUMBER_RANDOM).arrays()
    ref = O.read_hmsh(os.path.join(golden, "ref_import_wedge.hmsh"))
    for k in ("dim", "Nn", "Nc", "Nf", "Ncol", "NBCcol", "pnames"):
        assert m[k] == ref[k], k
    assert np.array_equal(np.diff(m["coloff"]), np.diff(ref["coloff"]))
    cells_a, faces_a = _canonical(m)
    cells_b, faces_b = _canonical(ref)
    assert cells_a == cells_b
    assert faces_a == faces_b and len(faces_a) == m["Nf"]


def test_wedge_command_writes_the_generated_mesh(tmp_path, capsys):
    """`python -m cfd_optimisations_b200.meshio wedge` writes the generator's mesh, readable by
    the library's checked reader and identical to the one the Python API builds."""
    out = tmp_path / "w.hmsh"
    meshio.main(["wedge", "41", "21", str(out), "--theta", "12", "--seed", "3", "--numbering", "rcm"])
    assert "1720 cells" in capsys.readouterr().out                    # 1,600 triangles + 120 ghosts
    a = H.Mesh(str(out)).arrays()
    b = H.Mesh.wedge(41, 21, theta_deg=12.0, seed=3, numbering=H.NUMBER_RCM).arrays()
    assert a["Nc"] == 2 * 40 * 20 + 2 * 40 + 2 * 20 and a["Nf"] == b["Nf"]
    for k in ("nodes", "fc_con", "fn_con", "cn_off", "cn_con", "coloff"):
        assert np.array_equal(a[k], b[k]), k
