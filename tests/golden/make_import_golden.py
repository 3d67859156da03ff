"""Regenerates the reference's own gmsh importer's outputs (interface/Mesh.py,
Mesh.generate_from_msh + write_hmsh, imported from the reference sources unchanged):

* ref_import_tri.hmsh — on the triangle-only rectangle that tests/test_meshio.py writes
  (write_msh(nx=9, ny=5, with_quads=False): 64 triangles, curves tagged 1..4);
* ref_import_wedge.hmsh — on the library's generated wedge (13 x 7 nodes, seed 3, random
  numbering) written as gmsh by write_msh_of_mesh (boundary colour k as curve tag k).

Run in a container that has the reference sources:

    python tests/golden/make_import_golden.py

The reference's importer imports matplotlib for its plotting functions, which are not used
here; matplotlib is absent from this image, so an empty stand-in module is registered
before the import.  The importer expects one element type and curve tags 1..n, so the
fixture mesh has only triangles.
"""
import importlib.util
import os
import sys
import tempfile
import types

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))


def reference_mesh_module():
    import oracle as O
    if "matplotlib" not in sys.modules:
        mpl = types.ModuleType("matplotlib")
        mpl.pyplot = types.ModuleType("matplotlib.pyplot")
        sys.modules["matplotlib"] = mpl
        sys.modules["matplotlib.pyplot"] = mpl.pyplot
    spec = importlib.util.spec_from_file_location("reference_mesh", os.path.join(O.REF_DIR, "interface", "Mesh.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def main():
    import cfd_optimisations_b200 as H
    from test_meshio import write_msh, write_msh_of_mesh
    R = reference_mesh_module()
    with tempfile.TemporaryDirectory() as tmp:
        src = os.path.join(tmp, "tri.msh")
        write_msh(src, nx=9, ny=5, with_quads=False)
        m = R.Mesh()
        m.generate_from_msh(src)
        m.write_hmsh(os.path.join(HERE, "ref_import_tri.hmsh"))
        src = os.path.join(tmp, "wedge.msh")
        write_msh_of_mesh(src, H.Mesh.wedge(13, 7, seed=3, numbering=H.NUMBER_RANDOM).arrays())
        m = R.Mesh()
        m.generate_from_msh(src)
        m.write_hmsh(os.path.join(HERE, "ref_import_wedge.hmsh"))


if __name__ == "__main__":
    main()
