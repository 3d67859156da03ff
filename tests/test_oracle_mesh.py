"""The oracle's wedge generator (oracle/hcfd_oracle_mesh.c), which writes the timed reference
arm's input without the product library, writes the same .hmsh bytes as the library's
generator for the same arguments, in every numbering."""
import filecmp

import pytest

import cfd_optimisations_b200 as H
import oracle as O


@pytest.mark.parametrize("numbering", [H.NUMBER_NATURAL, H.NUMBER_RANDOM, H.NUMBER_RCM, H.NUMBER_MORTON])
@pytest.mark.parametrize("nx,ny,theta,jitter,seed", [(41, 21, 15.0, 0.15, 1234), (161, 81, 15.0, 0.15, 1234),
                                                     (65, 33, 20.0, 0.1, 7), (33, 17, 0.0, 0.0, 3)])
def test_oracle_wedge_file_equals_the_library_file(tmp_path, numbering, nx, ny, theta, jitter, seed):
    a, b = str(tmp_path / "lib.hmsh"), str(tmp_path / "oracle.hmsh")
    H.Mesh.wedge(nx, ny, theta_deg=theta, jitter=jitter, seed=seed, numbering=numbering).write(a)
    O.wedge_hmsh(b, nx, ny, theta_deg=theta, jitter=jitter, seed=seed, numbering=numbering)
    assert filecmp.cmp(a, b, shallow=False)


def test_oracle_wedge_rejects_bad_arguments(tmp_path):
    with pytest.raises(ValueError):
        O.wedge_hmsh(str(tmp_path / "x.hmsh"), 2, 10)
    with pytest.raises(ValueError):
        O.wedge_hmsh(str(tmp_path / "x.hmsh"), 41, 21, jitter=0.6)
