"""Generate the golden fixtures under tests/golden/ from the reference itself.

sdk_cloud.ply + sdk_cloud_expected.npz: a 7-splat cloud written by the
reference Python SDK's GaussianCloud.save_ply (python/lumen/cloud.py:131-161)
and the values its load_ply (:163-199) reads back (columns x y z scale rot
opacity f_dc, "%.6f"), for the PLY reader's test.

capi_synthetic.npz: the splats the reference C library
(c_api/src/lumen_c.c:156-256, built into oracle/_ref/liblumen_ref.so by
``make -C oracle ref``) generates for lumen_create_synthetic_cube(4, 2.0) and
lumen_create_synthetic_sphere(128, 1.5), as [n, 59] float32 rows in
LumenGaussian field order.

sdk_depth_heatmap.npz: a 12 x 16 depth buffer holding the edge cases of the
SDK's depth visualisation (background at <= 0 and >= 999, the near and far
planes, values beyond them, infinities, NaN) plus seeded depths, and the RGB
bytes that the reference Python SDK's export_depth_visualization
(python/lumen/visualizer.py:16-48) writes for it with its default planes and
with near 1.25, far 7.5.

The reference source is needed only to run this script; the tests read the
committed files. Usage:

    python tests/golden/make_golden.py --reference <reference checkout> [capi] [ply] [depth]
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = os.path.join(ROOT, "oracle", "_ref", "liblumen_ref.so")


def main(reference: str):
    if not os.path.exists(REF):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "ref", f"REFERENCE={reference}"], check=True)
    lib = C.CDLL(REF)
    lib.lumen_create_synthetic_cube.restype = C.c_void_p
    lib.lumen_create_synthetic_cube.argtypes = [C.c_size_t, C.c_float]
    lib.lumen_create_synthetic_sphere.restype = C.c_void_p
    lib.lumen_create_synthetic_sphere.argtypes = [C.c_size_t, C.c_float]
    lib.lumen_cloud_get_count.restype = C.c_size_t
    lib.lumen_cloud_get_count.argtypes = [C.c_void_p]
    lib.lumen_cloud_get_gaussian.argtypes = [C.c_void_p, C.c_size_t, C.c_void_p]
    lib.lumen_cloud_destroy.argtypes = [C.c_void_p]

    def dump(cloud):
        n = lib.lumen_cloud_get_count(cloud)
        out = np.zeros((n, 59), np.float32)
        buf = (C.c_float * 59)()
        for i in range(n):
            lib.lumen_cloud_get_gaussian(cloud, i, buf)
            out[i] = np.frombuffer(buf, dtype=np.float32)
        lib.lumen_cloud_destroy(cloud)
        return out

    np.savez_compressed(os.path.join(HERE, "capi_synthetic.npz"),
                        cube_4_2=dump(lib.lumen_create_synthetic_cube(4, 2.0)),
                        **{"sphere_128_1.5": dump(lib.lumen_create_synthetic_sphere(128, 1.5))})


def sdk_ply(reference: str):
    """Needs the reference source tree (its Python SDK) on this machine."""
    import sys
    sys.path.insert(0, os.path.join(reference, "python"))
    from lumen.cloud import Gaussian3D, GaussianCloud
    rng = np.random.default_rng(7)
    cloud = GaussianCloud()
    for _ in range(7):
        q = rng.normal(size=4)
        q /= np.linalg.norm(q)
        sh = [0.0] * 48
        sh[:3] = [float(v) for v in rng.normal(0.5, 0.2, 3)]
        cloud.add(Gaussian3D(position=tuple(float(v) for v in rng.uniform(-2, 2, 3)),
                             scale=tuple(float(v) for v in rng.uniform(0.01, 0.3, 3)),
                             rotation=tuple(float(v) for v in q), opacity=float(rng.uniform(0.05, 1.0)),
                             sh_coeffs=sh))
    path = os.path.join(HERE, "sdk_cloud.ply")
    cloud.save_ply(path)
    back = GaussianCloud.load_ply(path)
    np.savez_compressed(os.path.join(HERE, "sdk_cloud_expected.npz"),
                        means=np.array([g.position for g in back.splats], np.float32),
                        scales=np.array([g.scale for g in back.splats], np.float32),
                        quats=np.array([g.rotation for g in back.splats], np.float32),
                        opacities=np.array([g.opacity for g in back.splats], np.float32),
                        sh=np.array([g.sh_coeffs for g in back.splats], np.float32))


def sdk_depth_heatmap(reference: str):
    """Needs the reference source tree (its Python SDK) on this machine."""
    import sys
    import tempfile
    sys.path.insert(0, os.path.join(reference, "python"))
    from lumen.visualizer import export_depth_visualization
    rng = np.random.default_rng(11)
    h, w = 12, 16
    d = rng.uniform(0.2, 12.0, h * w).astype(np.float32)
    edge = [0.0, -1.0, -0.0, 1e-4, 0.001, 0.5, 10.0, 998.99, 999.0, 1e4, np.inf, -np.inf, np.nan,
            0.4999, 10.0001, 5.25, 0.5 + 9.5 / 255.0, 3.0]
    d[:len(edge)] = np.array(edge, np.float32)
    d = d.reshape(h, w)
    out = {"depth": d}
    for tag, kw in (("default", {}), ("near1.25_far7.5", {"near_plane": 1.25, "far_plane": 7.5})):
        with tempfile.TemporaryDirectory() as tmp:
            path = os.path.join(tmp, "d.ppm")
            export_depth_visualization(path, w, h, [float(v) for v in d.reshape(-1)], **kw)
            raw = open(path, "rb").read()
        header = f"P6\n{w} {h}\n255\n".encode("ascii")
        assert raw.startswith(header)
        out[tag] = np.frombuffer(raw[len(header):], np.uint8).reshape(h, w, 3)
    np.savez_compressed(os.path.join(HERE, "sdk_depth_heatmap.npz"), **out)


if __name__ == "__main__":
    import argparse
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--reference", required=True, help="the reference checkout (its c_api/ and python/ trees)")
    ap.add_argument("which", nargs="*", default=["capi", "ply", "depth"])
    a = ap.parse_args()
    if "capi" in a.which:
        main(a.reference)
    if "ply" in a.which:
        sdk_ply(a.reference)
    if "depth" in a.which:
        sdk_depth_heatmap(a.reference)
