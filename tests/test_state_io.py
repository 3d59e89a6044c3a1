"""State I/O through the C ABI: the reference's LEVELSET_3D binary format
(read a file the reference wrote, write one the reference can read) and
checkpoint/resume of the whole step state."""
import os
import struct

import numpy as np
import pytest

import fluid_simulator_backup_b200 as fs

GOLD = os.path.join(os.path.dirname(__file__), "golden")
pytestmark = pytest.mark.gpu
HEADER = struct.Struct("<6i6di")  # LEVELSET_3D::Write: 6 int32, 6 float64, int32 ghost width


def load(name):
    return dict(np.load(os.path.join(GOLD, name + ".npz")))


def test_reads_a_levelset_written_by_the_reference(tmp_path):
    g = load("levelset_file")
    n = int(g["n"])
    path = tmp_path / "ref.bin"
    path.write_bytes(g["raw"].tobytes())
    with fs.Solver(n, float(g["dx"])) as s:
        mn = s.read_levelset(path)
        phi = s.download("phi")
    assert mn == (0.0, 0.0, 0.0)
    np.testing.assert_array_equal(phi, g["phi"])


def test_writes_the_reference_format(tmp_path):
    g = load("levelset_file")
    n = int(g["n"])
    ref = g["raw"].tobytes()
    path = tmp_path / "ours.bin"
    with fs.Solver(n, float(g["dx"])) as s:
        s.upload("phi", g["phi"])
        s.write_levelset(path)
    ours = path.read_bytes()
    assert len(ours) == len(ref)
    hi, hr = HEADER.unpack_from(ours), HEADER.unpack_from(ref)
    assert hi[:6] == hr[:6]
    # x_max = x_min + (n-1) dx here, (n-1)/n as parsed from the script in the reference
    np.testing.assert_allclose(hi[6:12], hr[6:12], rtol=1e-15)
    assert ours[HEADER.size:] == ref[HEADER.size:]


def test_rejects_a_levelset_of_another_grid(tmp_path):
    g = load("levelset_file")
    path = tmp_path / "ref.bin"
    path.write_bytes(g["raw"].tobytes())
    n = int(g["n"]) + 1
    with fs.Solver(n, 1.0 / n) as s:
        with pytest.raises(fs.FsError) as e:
            s.read_levelset(path)
        assert e.value.status == fs.FS_INVALID_ARG
        assert "level set" in str(e.value)
    truncated = tmp_path / "short.bin"
    truncated.write_bytes(g["raw"].tobytes()[:-8])
    with fs.Solver(int(g["n"]), float(g["dx"])) as s:
        with pytest.raises(fs.FsError):
            s.read_levelset(truncated)


def test_checkpoint_resume_reproduces_the_step(tmp_path):
    n = 12
    x = (np.arange(n) + 0.5) / n
    phi = np.sqrt((x[None, None, :] - 0.5) ** 2 + (x[None, :, None] - 0.4) ** 2 + (x[:, None, None] - 0.5) ** 2) - 0.25
    rng = np.random.default_rng(0)
    state = {"phi": phi, "u": rng.normal(size=(n, n, n + 1)) * 0.05, "v": rng.normal(size=(n, n + 1, n)) * 0.05,
             "w": rng.normal(size=(n + 1, n, n)) * 0.05}
    path = tmp_path / "state.bin"
    with fs.Solver(n, 1.0 / n, tolerance=1e-10, stop=fs.FS_STOP_RELATIVE) as a:
        for k, v in state.items():
            a.upload(k, v)
        dt = a.cfl_dt()
        a.step(dt)
        a.write_state(path)
        a.step(dt)
        want = {k: a.download(k) for k in ("phi", "u", "v", "w", "pressure")}
    with fs.Solver(n, 1.0 / n, tolerance=1e-10, stop=fs.FS_STOP_RELATIVE) as b:
        b.read_state(path)
        b.step(dt)
        got = {k: b.download(k) for k in ("phi", "u", "v", "w", "pressure")}
    for k in want:
        np.testing.assert_array_equal(got[k], want[k])
