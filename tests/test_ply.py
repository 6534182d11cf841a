"""PLY scenes (include/lumen_ply.h) on the host: header parsing, columns
by property name, SH transposition of the training layout, error codes.

The reference's two ASCII readers (src/scene/ply.mojo:73-138,
python/lumen/cloud.py:163-199) take columns by position in their own
writers' orders; here the reader maps them by name, and is pinned on a
file written by the reference SDK itself (tests/golden/sdk_cloud.ply).
"""
import os

import numpy as np
import pytest

from lumen_b200 import _lib as L
from lumen_b200 import ply

HERE = os.path.dirname(os.path.abspath(__file__))


def test_reference_sdk_file_reads_like_the_sdk(tmp_path):
    path = os.path.join(HERE, "golden", "sdk_cloud.ply")
    exp = np.load(os.path.join(HERE, "golden", "sdk_cloud_expected.npz"))
    inf = ply.info(path)
    assert inf.count == 7 and not inf.binary and inf.sh_degree == 0 and not inf.log_values
    a, _ = ply.load_host(path)
    for k in ("means", "scales", "quats", "opacities", "sh"):
        assert np.array_equal(a[k], exp[k].reshape(a[k].shape)), k


def write_mojo_ascii(path, means, scales, quats, opac, dc):
    """The column order of write_ply_ascii, src/scene/ply.mojo:32-70."""
    head = ["ply", "format ascii 1.0", "comment Created by Lumen 3D Gaussian Splatting Engine",
            f"element vertex {len(means)}"]
    head += [f"property float {n}" for n in ("x", "y", "z", "f_dc_0", "f_dc_1", "f_dc_2", "opacity", "scale_0",
                                             "scale_1", "scale_2", "rot_0", "rot_1", "rot_2", "rot_3")]
    head.append("end_header")
    with open(path, "w") as f:
        f.write("\n".join(head) + "\n")
        for i in range(len(means)):
            vals = [*means[i], *dc[i], opac[i], *scales[i], *quats[i]]
            f.write(" ".join(repr(float(v)) for v in vals) + "\n")


def test_mojo_layout_ascii(tmp_path):
    rng = np.random.default_rng(1)
    n = 50
    means = rng.uniform(-3, 3, (n, 3)).astype(np.float32)
    scales = rng.uniform(0.01, 0.2, (n, 3)).astype(np.float32)
    quats = rng.normal(size=(n, 4)).astype(np.float32)
    opac = rng.uniform(0, 1, n).astype(np.float32)
    dc = rng.normal(0.5, 0.2, (n, 3)).astype(np.float32)
    p = str(tmp_path / "mojo.ply")
    write_mojo_ascii(p, means, scales, quats, opac, dc)
    a, inf = ply.load_host(p)
    assert inf.count == n and inf.sh_degree == 0 and not inf.log_values
    assert np.array_equal(a["means"], means) and np.array_equal(a["scales"], scales)
    assert np.array_equal(a["quats"], quats) and np.array_equal(a["opacities"], opac)
    assert np.array_equal(a["sh"][:, :3], dc) and not a["sh"][:, 3:].any()


@pytest.mark.parametrize("degree,normals", [(3, True), (2, False), (1, True), (0, False)])
def test_training_layout_binary(tmp_path, degree, normals):
    rng = np.random.default_rng(degree)
    n = 1000
    means = rng.normal(size=(n, 3)).astype(np.float32)
    ls = rng.normal(-3, 0.5, (n, 3)).astype(np.float32)
    q = rng.normal(size=(n, 4)).astype(np.float32)
    logit = rng.normal(size=n).astype(np.float32)
    sh = rng.normal(size=(n, 16, 3)).astype(np.float32)
    p = str(tmp_path / "train.ply")
    ply.write_binary(p, means, ls, q, logit, sh, sh_degree=degree, normals=normals)
    inf = ply.info(p)
    m = (degree + 1) ** 2 - 1
    assert inf.binary and inf.sh_degree == degree and inf.count == n
    assert inf.log_values == (m > 0)
    assert inf.vertex_stride == 4 * (3 + 3 * normals + 3 + 3 * m + 1 + 3 + 4)
    a, _ = ply.load_host(p)
    assert np.array_equal(a["means"], means) and np.array_equal(a["scales"], ls)
    assert np.array_equal(a["quats"], q) and np.array_equal(a["opacities"], logit)
    want = sh.copy()
    want[:, m + 1:, :] = 0.0
    assert np.array_equal(a["sh"].reshape(n, 16, 3), want)


def test_values_override(tmp_path):
    p = str(tmp_path / "t.ply")
    z = np.zeros((3, 3), np.float32)
    ply.write_binary(p, z, z, np.tile([1, 0, 0, 0], (3, 1)), np.zeros(3), np.zeros((3, 48)), sh_degree=0)
    assert not ply.info(p).log_values
    assert ply.info(p, "log").log_values
    assert not ply.info(p, "linear").log_values


def test_unaligned_binary_and_extra_properties(tmp_path):
    """An 8-bit property between floats (colour bytes some tools add) is
    skipped by stride; the floats after it are unaligned and still read."""
    n = 20
    rng = np.random.default_rng(3)
    rows = rng.normal(size=(n, 14)).astype("<f4")
    names = ["x", "y", "z", "f_dc_0", "f_dc_1", "f_dc_2", "opacity", "scale_0", "scale_1", "scale_2",
             "rot_0", "rot_1", "rot_2", "rot_3"]
    head = "ply\nformat binary_little_endian 1.0\nelement vertex %d\n" % n
    head += "property float x\nproperty float y\nproperty float z\nproperty uchar red\n"
    head += "".join(f"property float {nm}\n" for nm in names[3:]) + "element face 0\nproperty list uchar int i\n"
    head += "end_header\n"
    body = b"".join(rows[i, :3].tobytes() + bytes([7]) + rows[i, 3:].tobytes() for i in range(n))
    p = str(tmp_path / "u.ply")
    with open(p, "wb") as f:
        f.write(head.encode() + body)
    inf = ply.info(p)
    assert inf.vertex_stride == 14 * 4 + 1
    a, _ = ply.load_host(p)
    assert np.array_equal(a["means"], rows[:, :3])
    assert np.array_equal(a["sh"][:, :3], rows[:, 3:6])
    assert np.array_equal(a["opacities"], rows[:, 6]) and np.array_equal(a["quats"], rows[:, 10:14])


def _status(path, values=0):
    c = L.LumenPlyInfo()
    return L.load().lumen_ply_info(str(path).encode(), values, c)


def test_errors(tmp_path):
    assert _status(tmp_path / "missing.ply") == -4                    # LUMEN_ERROR_IO_FAILURE
    bad = tmp_path / "bad.ply"
    bad.write_text("not a ply\n")
    assert _status(bad) == -1
    be = tmp_path / "be.ply"
    be.write_text("ply\nformat binary_big_endian 1.0\nelement vertex 1\nproperty float x\nend_header\n")
    assert _status(be) == -1
    noop = tmp_path / "noop.ply"
    props = "".join(f"property float {n}\n" for n in ("x", "y", "z", "scale_0", "scale_1", "scale_2", "rot_0",
                                                      "rot_1", "rot_2", "rot_3", "f_dc_0", "f_dc_1", "f_dc_2"))
    noop.write_text("ply\nformat ascii 1.0\nelement vertex 0\n" + props + "end_header\n")
    assert _status(noop) == -1                                        # no opacity column
    dbl = tmp_path / "dbl.ply"
    dbl.write_text("ply\nformat binary_little_endian 1.0\nelement vertex 0\n" +
                   props.replace("float x", "double x") + "property float opacity\nend_header\n")
    assert _status(dbl) == -1                                         # a mapped column not float32
    assert _status(tmp_path / "missing.ply", 3) == -1                 # bad values mode
    ok = tmp_path / "ok.ply"
    ok.write_text("ply\nformat ascii 1.0\nelement vertex 2\n" + props + "property float opacity\nend_header\n" +
                  "1 2 3 4 5 6 7 8 9 10 11 12 13 14\n")                # one vertex line missing
    arrs = [np.zeros(n, np.float32) for n in (6, 6, 8, 2, 96)]
    st = L.load().lumen_ply_load_host(str(ok).encode(), 0, *(a.ctypes.data for a in arrs), 2, None)
    assert st == -4
    st = L.load().lumen_ply_load_host(str(ok).encode(), 0, *(a.ctypes.data for a in arrs), 1, None)
    assert st == -1                                                   # capacity below the vertex count
