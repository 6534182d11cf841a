"""PLY scenes straight to the device (lumen_ply_load_device): the binary
training layout through the de-interleave kernel, unaligned binary and
ASCII files through the host parser, all equal to the host reader; a
loaded scene renders exactly like the same arrays uploaded by torch."""
import os

import numpy as np
import pytest

from lumen_b200 import ply, scenes
from lumen_b200.types import RenderOptions

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


def _same(scene, arrs):
    for k, t in zip(("means", "scales", "quats", "opacities", "sh"), scene.tensors):
        assert np.array_equal(t.cpu().numpy().reshape(arrs[k].shape), arrs[k]), k


def test_binary_training_layout_on_device(tmp_path):
    sc = scenes.box_scene(300_000, seed=9)
    p = str(tmp_path / "scene.ply")
    ply.write_binary(p, sc.means, sc.log_scales, sc.quats, sc.opacity_logits, sc.sh, sh_degree=3)
    dev, inf = ply.load(p)
    assert inf.binary and inf.log_values and inf.sh_degree == 3 and inf.count == sc.n
    host, _ = ply.load_host(p)
    _same(dev, host)
    # renders exactly like the arrays uploaded directly
    from lumen_b200 import render as R
    cam = scenes.camera_config1(640, 360)
    opt = RenderOptions(params_are_logits=True, term_mode=1)
    a = R.render(*dev.tensors, cam, opt)
    t = lambda x: torch.from_numpy(np.ascontiguousarray(x, np.float32)).cuda()
    b = R.render(t(sc.means), t(sc.log_scales), t(sc.quats), t(sc.opacity_logits).reshape(-1),
                 t(sc.sh).reshape(-1, 48), cam, opt)
    assert torch.equal(a.rgb, b.rgb) and torch.equal(a.n_contrib, b.n_contrib)


def test_ascii_and_unaligned_files_on_device(tmp_path):
    path = os.path.join(HERE, "golden", "sdk_cloud.ply")
    dev, inf = ply.load(path)
    host, _ = ply.load_host(path)
    assert not inf.binary and inf.count == 7
    _same(dev, host)
    n = 33
    rng = np.random.default_rng(5)
    rows = rng.normal(size=(n, 14)).astype("<f4")
    names = ["x", "y", "z", "f_dc_0", "f_dc_1", "f_dc_2", "opacity", "scale_0", "scale_1", "scale_2",
             "rot_0", "rot_1", "rot_2", "rot_3"]
    head = "ply\nformat binary_little_endian 1.0\nelement vertex %d\n" % n
    head += "property float x\nproperty float y\nproperty float z\nproperty uchar red\n"
    head += "".join(f"property float {nm}\n" for nm in names[3:]) + "end_header\n"
    body = b"".join(rows[i, :3].tobytes() + bytes([1]) + rows[i, 3:].tobytes() for i in range(n))
    p = str(tmp_path / "u.ply")
    with open(p, "wb") as f:
        f.write(head.encode() + body)
    dev, inf = ply.load(p)
    host, _ = ply.load_host(p)
    _same(dev, host)


def test_multi_chunk_binary(tmp_path):
    """More vertices than one 64 MB staging chunk (the two page-locked
    buffers alternate)."""
    n = 700_000          # 248 B per vertex with normals: about 2.6 chunks
    rng = np.random.default_rng(11)
    means = rng.normal(size=(n, 3)).astype(np.float32)
    ls = rng.normal(-3, 0.3, (n, 3)).astype(np.float32)
    q = rng.normal(size=(n, 4)).astype(np.float32)
    lg = rng.normal(size=n).astype(np.float32)
    sh = rng.normal(size=(n, 48)).astype(np.float32)
    p = str(tmp_path / "big.ply")
    ply.write_binary(p, means, ls, q, lg, sh)
    dev, inf = ply.load(p)
    assert inf.count == n
    host, _ = ply.load_host(p)
    _same(dev, host)
