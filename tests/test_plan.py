"""Host checks of the tiled kernels' execution plan (no GPU needed): every index the
kernels derive from the plan stays inside the staged range, each flux slot is written by
exactly one face entry, slots follow increasing face order, bulk copies are 16-byte sized."""
import os

import pytest

import cfd_optimisations_b200 as H


@pytest.mark.parametrize("numbering", [H.NUMBER_NATURAL, H.NUMBER_RANDOM, H.NUMBER_RCM, H.NUMBER_MORTON])
@pytest.mark.parametrize("keep", [False, True])
@pytest.mark.parametrize("tile", [32, 128, 256])
def test_plan_invariants_generated(numbering, keep, tile):
    m = H.Mesh.wedge(81, 41, seed=5, numbering=numbering)
    info = H.plan_check(m, tile=tile, keep_numbering=keep)
    assert info["slots"] == 3
    assert info["faces_once"] + info["faces_cut"] >= m.Nf


def test_plan_invariants_quads(golden):
    m = H.Mesh(os.path.join(golden, "wedge.hmsh"))
    for tile in (32, 64, 256):
        info = H.plan_check(m, tile=tile)
        assert info["slots"] == 4


def test_morton_tiles_are_compact():
    """Morton order keeps most faces inside one tile whatever the input numbering."""
    for numbering in (H.NUMBER_RANDOM, H.NUMBER_RCM):
        info = H.plan_check(H.Mesh.wedge(321, 161, seed=9, numbering=numbering))
        assert info["faces_cut"] / (info["faces_cut"] + info["faces_once"]) < 0.25
        assert info["halo_max"] < 128


def test_plan_rejects_bad_tile():
    m = H.Mesh.wedge(41, 21, seed=1)
    with pytest.raises(H.HcfdError):
        H.plan_check(m, tile=100000)
