"""Checkpoint file header checks on the CPU (hcfd_checkpoint_info reads no GPU state)."""
import struct

import pytest

import cfd_optimisations_b200 as H
from cfd_optimisations_b200.native import HcfdError

HDR = "<8siiiiqdddii"   # magic, version, precision, Nc, has_limiter, steps, res2 first/last, dt, nonfinite, pad


def write(path, Nc=5, precision=H.FP64, has_phi=0, steps=7, magic=b"HCFDCKP1", version=1, body=None):
    with open(path, "wb") as fh:
        fh.write(struct.pack(HDR, magic, version, precision, Nc, has_phi, steps, 1.0, 0.5, 1e-3, 0, 0))
        fh.write(body if body is not None else bytes(8 * 4 * Nc * (1 + has_phi)))


def test_header_size():
    assert struct.calcsize(HDR) == 64


def test_info_reads_header(tmp_path):
    p = tmp_path / "a.ckpt"
    write(p, Nc=11, precision=H.FP32, has_phi=1, steps=1234)
    assert H.checkpoint_info(str(p)) == dict(Nc=11, precision=H.FP32, steps=1234, has_limiter=True)


@pytest.mark.parametrize("kw", [dict(magic=b"HCFDCKP2"), dict(version=2), dict(Nc=0), dict(precision=7),
                                dict(has_phi=3), dict(steps=-1)])
def test_info_rejects_bad_headers(tmp_path, kw):
    p = tmp_path / "b.ckpt"
    write(p, **kw)
    with pytest.raises(HcfdError) as e:
        H.checkpoint_info(str(p))
    assert e.value.code == H.native.EIO


def test_info_rejects_missing_and_short_files(tmp_path):
    with pytest.raises(HcfdError):
        H.checkpoint_info(str(tmp_path / "missing.ckpt"))
    p = tmp_path / "short.ckpt"
    p.write_bytes(b"HCFDCKP1\x01\x00")
    with pytest.raises(HcfdError):
        H.checkpoint_info(str(p))
