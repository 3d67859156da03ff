"""Checkpoint file header checks on the CPU (hcfd_checkpoint_info reads no GPU state)."""
import struct

import numpy as np
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


def test_convert_checkpoint_to_fp32_rounds_values_and_sets_precision(tmp_path):
    """An FP64 checkpoint converted for an FP32 solver: same header but the precision, every
    value rounded to the nearest float (what an FP32 solver holds and writes)."""
    Nc = 6
    rng = np.random.default_rng(1)
    vals = rng.standard_normal(8 * Nc) * 1e3
    vals[0] = np.pi
    src, dst = tmp_path / "a64.ckpt", tmp_path / "a32.ckpt"
    write(src, Nc=Nc, precision=H.FP64, has_phi=1, steps=100, body=vals.astype("<f8").tobytes())
    info = H.convert_checkpoint(str(src), str(dst), H.FP32)
    assert info == dict(Nc=Nc, precision=H.FP32, steps=100, has_limiter=True)
    raw_src, raw_dst = src.read_bytes(), dst.read_bytes()
    assert len(raw_dst) == len(raw_src)
    assert raw_dst[:12] == raw_src[:12] and raw_dst[16:64] == raw_src[16:64]     # only the precision field changes
    out = np.frombuffer(raw_dst, dtype="<f8", offset=64)
    assert np.array_equal(out, vals.astype(np.float32).astype(np.float64))
    assert out[0] != np.pi and out[0] == np.float64(np.float32(np.pi))
    # back to FP64: values kept
    back = tmp_path / "b64.ckpt"
    assert H.convert_checkpoint(str(dst), str(back), H.FP64)["precision"] == H.FP64
    assert np.array_equal(np.frombuffer(back.read_bytes(), dtype="<f8", offset=64), out)


def test_convert_checkpoint_rejects_bad_input(tmp_path):
    src = tmp_path / "s.ckpt"
    write(src, Nc=4, body=bytes(8 * 4 * 4 - 8))                # one value short
    with pytest.raises(HcfdError):
        H.convert_checkpoint(str(src), str(tmp_path / "d.ckpt"), H.FP32)
    write(src, Nc=4)
    with pytest.raises(ValueError):
        H.convert_checkpoint(str(src), str(tmp_path / "d.ckpt"), 5)
    assert not (tmp_path / "d.ckpt").exists()
