"""Checkpoint files (fvm_save_checkpoint / fvm_load_checkpoint): header
validation on the CPU; on the GPU, a restored solve continues bit for bit
like the uninterrupted one, under both dt policies, Euler and NS."""
import struct
import zlib

import numpy as np
import pytest

from helpers import small
import fvm_b200
from fvm_b200 import abi


def _file(path, nx=8, ny=4, magic=b"FVMB200C", corrupt=False, version=1):
    p, e = small("euler_m3_circle", nx, ny)
    payload = np.arange(5 * nx * ny, dtype=np.float32).tobytes()
    head = bytearray(256)
    head[:8] = magic
    struct.pack_into("<IIiiII", head, 8, version, 256, nx, ny, 5, 0)
    struct.pack_into("<ffff", head, 32, 1e-6, 0.0, 0.0, 0.0)
    struct.pack_into("<QI", head, 48, len(payload), zlib.crc32(payload))
    head[64:64 + 112] = bytes(p)
    head[176:176 + len(bytes(e))] = bytes(e)
    if corrupt:
        payload = payload[:-1] + b"\x01"
    path.write_bytes(bytes(head) + payload)
    return path


def _info_status(path):
    lib = fvm_b200.load_library()
    return lib.fvm_checkpoint_info(str(path).encode(), None, None), lib.fvm_last_error()


def test_python_reader_and_header_checks(tmp_path):
    good = _file(tmp_path / "good.ckpt")
    hd, U = fvm_b200.read_checkpoint(good)
    assert U.shape == (5, 4, 8) and U[4, 3, 7] == 5 * 32 - 1
    assert hd["params"].nx == 8 and hd["next_dt"] == pytest.approx(1e-6)
    with pytest.raises(fvm_b200.FvmError):
        fvm_b200.read_checkpoint(_file(tmp_path / "bad.ckpt", corrupt=True))


@pytest.mark.parametrize("kind, msg", [("magic", b"not a checkpoint"), ("corrupt", b"checksum"),
                                       ("version", b"unsupported")])
def test_library_validates_files_without_a_device(tmp_path, kind, msg):
    kw = {"magic": {"magic": b"NOTACKPT"}, "corrupt": {"corrupt": True}, "version": {"version": 9}}[kind]
    rc, err = _info_status(_file(tmp_path / "x.ckpt", **kw))
    assert rc in (1, 8) and msg in err
    p, _ = fvm_b200.checkpoint_info(_file(tmp_path / "ok.ckpt"))
    assert (p.nx, p.ny) == (8, 4)


@pytest.mark.gpu
@pytest.mark.parametrize("policy", [abi.DT_FIXED, abi.DT_RECOMPUTE])
@pytest.mark.parametrize("case", [("euler_m3_circle", 160, 80), ("ns_karman_re200", 160, 80)])
def test_restored_solve_continues_bitwise(tmp_path, policy, case):
    p, e = small(*case)
    e.dt_policy = policy
    s = fvm_b200.Solver(p, e)
    if policy == abi.DT_FIXED:
        s.params.dt = s.compute_dt()
    s.step(11)
    path = tmp_path / "s.ckpt"
    s.save_checkpoint(path)
    hd, U = fvm_b200.read_checkpoint(path)
    assert np.array_equal(U.view(np.uint32), s.fields().view(np.uint32))
    s.step(9)
    a, ta = s.fields(), s.params.t_current
    s2 = fvm_b200.Solver()
    q = s2.load_checkpoint(path)
    assert q.step == 11
    s2.step(9)
    assert np.array_equal(a.view(np.uint32), s2.fields().view(np.uint32))
    assert s2.params.t_current == ta and s2.params.step == 20
