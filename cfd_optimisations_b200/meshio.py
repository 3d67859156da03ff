"""Mesh import and solution export: gmsh .msh (version 4.1, ASCII) to .hmsh, and .hsln solutions
to VTK .vtu files, as the reference's `HCFD import` / `export` / `bexport` / `checkcell` commands
do (interface/Mesh.py, interface/Export.py), without its matplotlib and vtk dependencies.

Import (2-D): every surface element (triangle, quadrangle) is a real cell; every line element on
a curve that carries a physical tag is a ghost cell of that tag's boundary colour.  Cells that
share an edge are neighbours; each shared edge is a face.  Colour 0 holds the interior faces,
colours 1..n the boundary faces of the physical curve tags in increasing order (coltag[c] = c,
as the reference writes them), each boundary face with its real cell on the left and its ghost
on the right.  Interior faces have the lower cell number on the left.  Faces are ordered by colour,
then by (left, right).  Cells are numbered by reverse Cuthill-McKee on the cell graph (scipy),
nodes by their first appearance in the renumbered cells.  The physical names kept are those of
the boundary curves, in colour order (the names the reference's reader exposes).

Export writes an UnstructuredGrid .vtu with inline base64 binary arrays: points (z = 0), cells
(triangle, quad and line cells with VTK types 5, 9, 3), and one cell array per solution variable,
the velocity components combined into one 3-component vector "Velocity", as the reference's
exporter names them.

`wedge NX NY OUT` writes the library's generated supersonic wedge (hcfd_mesh_generate_wedge)
as .hmsh, the mesh family of the workloads, without gmsh.
"""
from __future__ import annotations

import argparse
import base64
import glob
import re
import struct

import numpy as np

GMSH_NODES = {1: 2, 2: 3, 3: 4}           # element type -> nodes (line, triangle, quadrangle)
VTK_TYPE = {1: 3, 2: 5, 3: 9}             # gmsh element type -> VTK cell type


class MshError(ValueError):
    pass


def _sections(text: str) -> dict:
    out = {}
    for m in re.finditer(r"^\$(\w+)\s*$(.*?)^\$End\1\s*$", text, re.S | re.M):
        out[m.group(1)] = m.group(2).split()
    return out


def read_msh(path: str) -> dict:
    """Parses a gmsh 4.1 ASCII file into nodes, element blocks and physical names/tags."""
    with open(path, "r") as fh:
        text = fh.read()
    sec = _sections(text)
    fmt = sec.get("MeshFormat")
    if not fmt or not fmt[0].startswith("4.") or fmt[1] != "0":
        raise MshError(f"{path}: only gmsh 4.x ASCII files are read")
    # physical names: dim tag "name"
    names = {}
    pn = re.search(r"^\$PhysicalNames\s*$(.*?)^\$EndPhysicalNames", text, re.S | re.M)
    if pn:
        for line in pn.group(1).strip().splitlines()[1:]:
            m = re.match(r"\s*(\d+)\s+(\d+)\s+\"(.*)\"", line)
            if m:
                names[(int(m.group(1)), int(m.group(2)))] = m.group(3)
    # entities: physical tag of each curve and surface
    ent = [float(x) for x in sec["Entities"]]
    k = 0
    npt, ncu, nsu, nvo = (int(x) for x in ent[0:4])
    k = 4
    if nvo:
        raise MshError(f"{path}: 3-D meshes are not supported")
    if nsu == 0:
        raise MshError(f"{path}: no surface")
    for _ in range(npt):                                   # tag x y z nphys phys...
        nph = int(ent[k + 4])
        k += 5 + nph
    curve_phys = {}
    for _ in range(ncu):                                   # tag box(6) nphys phys... nbound bound...
        tag, nph = int(ent[k]), int(ent[k + 7])
        phys = [int(x) for x in ent[k + 8:k + 8 + nph]]
        if len(phys) > 1:
            raise MshError(f"{path}: curve {tag} has more than one physical tag")
        curve_phys[tag] = phys[0] if phys else None
        nb = int(ent[k + 8 + nph])
        k += 9 + nph + nb
    # nodes
    nd = sec["Nodes"]
    nblocks, nnodes = int(nd[0]), int(nd[1])
    tags = np.empty(nnodes, dtype=np.int64)
    xyz = np.empty((nnodes, 3))
    k, h = 4, 0
    for _ in range(nblocks):
        parametric, n = int(nd[k + 2]), int(nd[k + 3])
        if parametric:
            raise MshError(f"{path}: parametric nodes are not supported")
        tags[h:h + n] = np.array(nd[k + 4:k + 4 + n], dtype=np.int64)
        xyz[h:h + n] = np.array(nd[k + 4 + n:k + 4 + 4 * n], dtype=np.float64).reshape(n, 3)
        k += 4 + 4 * n
        h += n
    # elements: (dim, entity, type, node tags [n, nn])
    el = sec["Elements"]
    nblocks = int(el[0])
    blocks = []
    k = 4
    for _ in range(nblocks):
        edim, etag, etype, n = (int(x) for x in el[k:k + 4])
        if etype not in GMSH_NODES:
            raise MshError(f"{path}: element type {etype} is not supported (lines, triangles, quadrangles)")
        nn = GMSH_NODES[etype]
        a = np.array(el[k + 4:k + 4 + n * (1 + nn)], dtype=np.int64).reshape(n, 1 + nn)
        blocks.append((edim, etag, etype, a[:, 1:]))
        k += 4 + n * (1 + nn)
    return dict(node_tags=tags, xyz=xyz, blocks=blocks, curve_phys=curve_phys, names=names)


def build_mesh(msh: dict) -> dict:
    """The .hmsh arrays of a parsed gmsh mesh (see the module docstring for the conventions)."""
    from scipy.sparse import coo_matrix
    from scipy.sparse.csgraph import reverse_cuthill_mckee

    index = {int(t): i for i, t in enumerate(msh["node_tags"])}
    cells, ctype, ptag = [], [], []
    for edim, etag, etype, conn in msh["blocks"]:
        if edim == 2:
            tag = 0
        elif edim == 1:
            tag = msh["curve_phys"].get(etag)
            if tag is None:
                raise MshError(f"line elements on curve {etag}, which has no physical tag")
            if tag <= 0:
                raise MshError(f"physical tag {tag} of curve {etag}: boundary tags must be positive")
        else:
            continue
        for row in conn:
            cells.append([index[int(x)] for x in row])
            ctype.append(etype)
            ptag.append(tag)
    nc = len(cells)
    ptag = np.array(ptag)
    # edges -> the cells that hold them
    owners = {}
    for c, nodes in enumerate(cells):
        k = len(nodes)
        if k == 2:
            e = (min(nodes), max(nodes))
            owners.setdefault(e, []).append(c)
            continue
        for j in range(k):
            a, b = nodes[j], nodes[(j + 1) % k]
            owners.setdefault((min(a, b), max(a, b)), []).append(c)
    pairs = []
    for e, cs in owners.items():
        if len(cs) == 1:
            if ptag[cs[0]] == 0:
                raise MshError(f"boundary edge {e} has no line element on a physical curve")
            continue
        if len(cs) != 2:
            raise MshError(f"edge {e} is shared by {len(cs)} cells")
        pairs.append((cs[0], cs[1], e))
    # cell numbering: reverse Cuthill-McKee on the cell graph
    r = np.array([p[0] for p in pairs] + [p[1] for p in pairs])
    c = np.array([p[1] for p in pairs] + [p[0] for p in pairs])
    g = coo_matrix((np.ones(len(r), dtype=np.int8), (r, c)), shape=(nc, nc)).tocsr()
    perm = np.asarray(reverse_cuthill_mckee(g, symmetric_mode=True), dtype=np.int64)
    new = np.empty(nc, dtype=np.int64)
    new[perm] = np.arange(nc)
    # node numbering: first appearance in the renumbered cells
    nnew = -np.ones(len(index), dtype=np.int64)
    nxt = 0
    for oc in perm:
        for n in cells[oc]:
            if nnew[n] < 0:
                nnew[n] = nxt
                nxt += 1
    if nxt != len(index):
        raise MshError("nodes that belong to no cell")
    # faces
    bc_tags = sorted(set(int(t) for t in ptag if t > 0))
    colour_of = {0: 0, **{t: i + 1 for i, t in enumerate(bc_tags)}}
    faces = []
    for a, b, (n1, n2) in pairs:
        A, B = int(new[a]), int(new[b])
        ta, tb = ptag[a], ptag[b]
        if ta > 0 and tb > 0:
            raise MshError("two boundary line elements share an edge")
        if ta > 0:
            A, B = B, A                                  # ghost on the right
        elif tb == 0 and A > B:
            A, B = B, A                                  # interior: lower number on the left
        col = colour_of[int(max(ta, tb))]
        m1, m2 = sorted((int(nnew[n1]), int(nnew[n2])))
        faces.append((col, A, B, m1, m2))
    faces.sort()
    F = np.array(faces, dtype=np.int64).reshape(-1, 5)
    ncol = len(bc_tags) + 1
    coloff = np.searchsorted(F[:, 0], np.arange(ncol + 1)).astype(np.int32)
    # cells in the new order
    cn_off = np.zeros(nc + 1, dtype=np.int32)
    cn_con, ctypes = [], np.empty(nc, dtype=np.int32)
    for i, oc in enumerate(perm):
        cn_con.extend(int(nnew[n]) for n in cells[oc])
        cn_off[i + 1] = len(cn_con)
        ctypes[i] = ctype[oc]
    nbr = [[] for _ in range(nc)]
    for _, A, B, _, _ in faces:
        nbr[A].append(B)
        nbr[B].append(A)
    cc_off = np.zeros(nc + 1, dtype=np.int32)
    cc_con = []
    for i in range(nc):
        cc_con.extend(sorted(nbr[i]))
        cc_off[i + 1] = len(cc_con)
    nodes = np.empty((len(index), 2))
    nodes[nnew] = msh["xyz"][:, :2]
    pnames = [msh["names"].get((1, t), f"boundary_{t}") for t in bc_tags]
    return dict(dim=2, Nn=len(index), Ncol=ncol, NBCcol=ncol - 1, Nc=nc, Nf=len(faces), pnames=pnames,
                coltag=np.arange(ncol, dtype=np.int32), coloff=coloff, nodes=nodes.ravel(),
                fn_con=F[:, 3:5].astype(np.int32).ravel(), fc_con=F[:, 1:3].astype(np.int32).ravel(),
                cn_off=cn_off, cn_con=np.array(cn_con, dtype=np.int32), cc_off=cc_off,
                cc_con=np.array(cc_con, dtype=np.int32), c_ctypes=ctypes)


def write_hmsh(path: str, m: dict) -> None:
    """The .hmsh layout src/Mesh.cpp:7-54 reads (8 int32 counts, the names, then the arrays), and
    the c_ctypes array interface/Mesh.py:441-463 appends."""
    names = b"".join(n.encode() + b"\0" for n in m["pnames"])
    with open(path, "wb") as fh:
        fh.write(struct.pack("<8i", m["dim"], m["Nn"], m["Ncol"], m["NBCcol"], m["Nc"], m["Nf"],
                             len(m["pnames"]), len(names)))
        fh.write(names)
        for key, dt in (("coltag", np.int32), ("coloff", np.int32), ("nodes", np.float64), ("fn_con", np.int32),
                        ("fc_con", np.int32), ("cn_off", np.int32), ("cn_con", np.int32), ("cc_off", np.int32),
                        ("cc_con", np.int32), ("c_ctypes", np.int32)):
            fh.write(np.ascontiguousarray(m[key], dtype=dt).tobytes())


def import_msh(msh_path: str, hmsh_path: str) -> dict:
    m = build_mesh(read_msh(msh_path))
    write_hmsh(hmsh_path, m)
    return m


def read_hsln(path: str):
    """A .hsln solution (src/Writer.cpp:22-39): names and an nvars x Nc array."""
    with open(path, "rb") as fh:
        b = fh.read()
    nc, nv, nch = struct.unpack_from("<3i", b, 0)
    names = [s.decode() for s in b[12:12 + nch].split(b"\0")[:-1]]
    data = np.frombuffer(b, dtype=np.float64, count=nv * nc, offset=12 + nch).reshape(nv, nc)
    return names, data.copy()


def _b64(a: np.ndarray) -> str:
    raw = np.ascontiguousarray(a).tobytes()
    return base64.b64encode(struct.pack("<I", len(raw)) + raw).decode()


def write_vtu(path: str, mesh: dict, names, data: np.ndarray) -> None:
    """Writes the cells of `mesh` (the arrays of Mesh.arrays() or build_mesh) with cell data."""
    nc = int(mesh["Nc"])
    nodes = np.asarray(mesh["nodes"], dtype=np.float64).reshape(-1, 2)
    pts = np.hstack([nodes, np.zeros((len(nodes), 1))])
    off = np.asarray(mesh["cn_off"], dtype=np.int64)
    ctypes = mesh.get("c_ctypes")
    if ctypes is None:
        ctypes = np.where(np.diff(off) == 2, 1, np.where(np.diff(off) == 3, 2, 3))
    types = np.array([VTK_TYPE[int(t)] for t in ctypes], dtype=np.uint8)
    arrays = []
    vel = [i for i, n in enumerate(names) if "velocity" in n.lower()]
    for i, n in enumerate(names):
        if i in vel:
            continue
        arrays.append((n, 1, np.asarray(data[i], dtype=np.float64)))
    if vel:
        v = np.zeros((nc, 3))
        for j, i in enumerate(vel[:3]):
            v[:, j] = data[i]
        arrays.append(("Velocity", 3, v))
    cell_xml = "".join(
        f'<DataArray type="Float64" Name="{n}" NumberOfComponents="{k}" format="binary">{_b64(a)}</DataArray>'
        for n, k, a in arrays)
    with open(path, "w") as fh:
        fh.write('<?xml version="1.0"?>\n<VTKFile type="UnstructuredGrid" version="1.0" byte_order="LittleEndian" '
                 'header_type="UInt32">\n<UnstructuredGrid>\n'
                 f'<Piece NumberOfPoints="{len(pts)}" NumberOfCells="{nc}">\n'
                 f'<Points><DataArray type="Float64" NumberOfComponents="3" format="binary">{_b64(pts)}'
                 '</DataArray></Points>\n<Cells>'
                 f'<DataArray type="Int64" Name="connectivity" format="binary">'
                 f'{_b64(np.asarray(mesh["cn_con"], dtype=np.int64))}</DataArray>'
                 f'<DataArray type="Int64" Name="offsets" format="binary">{_b64(off[1:])}</DataArray>'
                 f'<DataArray type="UInt8" Name="types" format="binary">{_b64(types)}</DataArray></Cells>\n'
                 f'<CellData>{cell_xml}</CellData>\n</Piece>\n</UnstructuredGrid>\n</VTKFile>\n')


def export(mesh_path: str, hsln_path: str, vtu_path: str) -> None:
    from . import Mesh
    m = Mesh(mesh_path).arrays()
    names, data = read_hsln(hsln_path)
    if data.shape[1] != m["Nc"]:
        raise ValueError(f"{hsln_path}: {data.shape[1]} cells, the mesh has {m['Nc']}")
    write_vtu(vtu_path, m, names, data)


def batch_export(mesh_path: str, in_pattern: str, out_pattern: str, quiet: bool = False) -> list:
    """Exports every file matching `in_pattern` (with %d for the snapshot number) to
    `out_pattern` with the same number."""
    from . import Mesh
    m = Mesh(mesh_path).arrays()
    rx = re.compile(re.escape(in_pattern).replace("%d", r"(\d+)") + "$")
    done = []
    for p in sorted(glob.glob(in_pattern.replace("%d", "*"))):
        hit = rx.search(p)
        if not hit:
            if not quiet:
                print(f"skipping {p}: does not match {in_pattern}")
            continue
        names, data = read_hsln(p)
        out = out_pattern.replace("%d", hit.group(1))
        write_vtu(out, m, names, data)
        done.append(out)
    return done


def check_cell(mesh_path: str, cell: int) -> dict:
    from . import Mesh
    m = Mesh(mesh_path).arrays()
    a, b = m["cn_off"][cell], m["cn_off"][cell + 1]
    nodes = m["cn_con"][a:b]
    xy = np.asarray(m["nodes"]).reshape(-1, 2)[nodes]
    nb = m["cc_con"][m["cc_off"][cell]:m["cc_off"][cell + 1]] if m.get("cc_off") is not None else []
    return dict(cell=cell, type=int(m["c_ctypes"][cell]) if m.get("c_ctypes") is not None else None,
                nodes=[int(x) for x in nodes], neighbours=[int(x) for x in nb], centre=xy.mean(axis=0).tolist())


def main(argv=None):
    ap = argparse.ArgumentParser(prog="hcfd", description="mesh import and solution export")
    sp = ap.add_subparsers(dest="cmd", required=True)
    p = sp.add_parser("import", help="gmsh .msh (4.1 ASCII) -> .hmsh")
    p.add_argument("meshin")
    p.add_argument("meshout")
    p = sp.add_parser("export", help=".hsln -> .vtu")
    p.add_argument("mesh")
    p.add_argument("solnin")
    p.add_argument("solnout")
    p = sp.add_parser("bexport", help="many .hsln -> .vtu (%%d in the patterns)")
    p.add_argument("mesh")
    p.add_argument("solnin_pattern")
    p.add_argument("solnout_pattern")
    p.add_argument("-Wnone", action="store_true", help="no warnings for files that do not match")
    p = sp.add_parser("checkcell", help="one cell's type, nodes, neighbours and centre")
    p.add_argument("meshin")
    p.add_argument("cell", type=int)
    p = sp.add_parser("wedge", help="generate a triangulated supersonic wedge -> .hmsh")
    p.add_argument("nx", type=int)
    p.add_argument("ny", type=int)
    p.add_argument("meshout")
    p.add_argument("--theta", type=float, default=15.0, help="ramp angle, degrees")
    p.add_argument("--jitter", type=float, default=0.15, help="interior node jitter, fraction of the spacing")
    p.add_argument("--seed", type=int, default=1234)
    p.add_argument("--numbering", choices=["natural", "random", "rcm", "morton"], default="random")
    a = ap.parse_args(argv)
    if a.cmd == "import":
        import_msh(a.meshin, a.meshout)
    elif a.cmd == "export":
        export(a.mesh, a.solnin, a.solnout)
    elif a.cmd == "bexport":
        batch_export(a.mesh, a.solnin_pattern, a.solnout_pattern, a.Wnone)
    elif a.cmd == "wedge":
        import cfd_optimisations_b200 as H
        num = {"natural": H.NUMBER_NATURAL, "random": H.NUMBER_RANDOM, "rcm": H.NUMBER_RCM,
               "morton": H.NUMBER_MORTON}[a.numbering]
        m = H.Mesh.wedge(a.nx, a.ny, theta_deg=a.theta, jitter=a.jitter, seed=a.seed, numbering=num)
        m.write(a.meshout)
        print(f"{a.meshout}: {m.Nc} cells, {m.Nf} faces")
    else:
        print(check_cell(a.meshin, a.cell))


if __name__ == "__main__":
    main()
