"""The reference's own test programs, unmodified, against the drop-ins.

* c_api/test/test_c_api.c, compiled against the reference's own lumen.h and
  linked to lumen_b200/liblumen.so (oracle/Makefile, target
  _ref/test_c_api_lumen_b200). Its last test, test_rasterization_pipeline
  (test_c_api.c:127-172: a 64-splat cube at 160x120 through lumen_rasterize),
  needs the GPU; the five before it are host-side.
* python/tests/test_client.py, run with ``lumen`` bound to lumen_b200 in
  sys.modules. TestLumenCamera and TestLumenCloud are host-side;
  TestLumenEngine renders through liblumen.so on the GPU.

Both files are placed under oracle/_ref by ``make -C oracle ref`` (which
build() runs where the reference checkout exists); the tests skip when that
build step did not run.
"""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
C_HARNESS = os.path.join(ROOT, "oracle", "_ref", "test_c_api_lumen_b200")
SDK_TESTS = os.path.join(ROOT, "oracle", "_ref", "sdk_tests")

HOST_C_TESTS = ("test_version", "test_config", "test_cloud_lifecycle", "test_synthetic_scenes", "test_framebuffer")
HOST_SDK_CLASSES = ("TestLumenCamera", "TestLumenCloud")

# unittest over the unmodified module, `lumen` resolved to lumen_b200
_RUNNER = """
import sys, unittest
sys.path[:0] = [{root!r}, {tests!r}]
import lumen_b200
sys.modules["lumen"] = lumen_b200
names = sys.argv[1:]
suite = (unittest.defaultTestLoader.loadTestsFromNames(["test_client." + n for n in names]) if names
         else unittest.defaultTestLoader.loadTestsFromName("test_client"))
res = unittest.TextTestRunner(verbosity=2).run(suite)
sys.exit(0 if res.wasSuccessful() and res.testsRun > 0 else 1)
"""


def _need(path):
    if not os.path.exists(path):
        pytest.skip(f"{os.path.relpath(path, ROOT)} not built (make -C oracle ref REFERENCE=...)")


def run_c_harness():
    _need(C_HARNESS)
    return subprocess.run([C_HARNESS], capture_output=True, text=True, timeout=300)


def run_sdk_tests(classes=()):
    _need(os.path.join(SDK_TESTS, "test_client.py"))
    code = _RUNNER.format(root=ROOT, tests=SDK_TESTS)
    return subprocess.run([sys.executable, "-c", code, *classes], capture_output=True, text=True, timeout=600,
                          cwd=ROOT)


def test_c_harness_links_this_library():
    _need(C_HARNESS)
    out = subprocess.run(["ldd", C_HARNESS], capture_output=True, text=True).stdout
    line = next(l for l in out.splitlines() if "liblumen.so" in l)
    assert os.path.realpath(line.split("=>")[1].split("(")[0].strip()) == \
        os.path.realpath(os.path.join(ROOT, "lumen_b200", "liblumen.so"))


def test_c_harness_host_tests():
    """The host-side half of test_c_api.c passes against liblumen.so (on a
    machine without a device the program stops at the rasterizer)."""
    r = run_c_harness()
    for name in HOST_C_TESTS:
        assert f"[PASS] {name}" in r.stdout, r.stdout


def test_sdk_host_tests_unmodified():
    r = run_sdk_tests(HOST_SDK_CLASSES)
    assert r.returncode == 0, r.stdout + r.stderr


@pytest.mark.gpu
def test_c_harness_all_assertions_on_gpu():
    r = run_c_harness()
    assert r.returncode == 0, r.stdout + r.stderr
    assert "[PASS] test_rasterization_pipeline" in r.stdout
    assert "100% SUCCESS" in r.stdout


@pytest.mark.gpu
def test_sdk_tests_unmodified_on_gpu():
    r = run_sdk_tests()
    assert r.returncode == 0, r.stdout + r.stderr
    assert "test_rasterize_scene" in r.stderr and "test_image_export" in r.stderr
