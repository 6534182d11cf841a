"""The render server (include/lumen_serve.h): continuous batching over
resident scenes.

Every served image must equal rendering its view alone (bit for bit, as
the 8-bit conversion of the standalone float render), whatever batch it
landed in: mixed scenes and resolutions, concurrent submitters, graph and
plain launches, every launch variant, and batches re-run after exceeding
their instance estimate.
"""
import threading

import numpy as np
import pytest

from lumen_b200 import scenes
from lumen_b200.types import RenderOptions, ViewCamera

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

OPT = RenderOptions(term_mode=1)


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).cuda()


def device_scene(sc):
    from lumen_b200 import render as R
    s, op = sc.activated()
    return R.Scene(_dev(sc.means), _dev(s), _dev(sc.quats), _dev(op).reshape(-1), _dev(sc.sh).reshape(-1, 48))


def alone_u8(scene, cam, opt=OPT):
    """The request rendered by itself through the plain forward, as bytes
    (uint8)(clamp(c, 0, 1) * 255)."""
    from lumen_b200 import render as R
    r = R.render(*scene.tensors, cam, opt)
    return (r.rgb.clamp(0.0, 1.0) * 255.0).to(torch.uint8).cpu()


@pytest.fixture(scope="module")
def world():
    sc = [device_scene(scenes.box_scene(n, seed=40 + i)) for i, n in enumerate((3000, 20_000, 60_000))]
    cams = []
    for i, (w, h) in enumerate(((160, 120), (320, 180), (97, 61), (640, 360))):
        cams += scenes.orbit_cameras(3, w, h, radius=9.0 + i, phase=0.3 * i)
    reqs = [(i % 3, cams[(5 * i) % len(cams)]) for i in range(24)]
    refs = [alone_u8(sc[s], c) for s, c in reqs]
    return sc, reqs, refs


def serve_all(server, sc, reqs, stagger=False):
    from lumen_b200 import serve
    ids = [server.add_scene(s) for s in sc]
    out = []
    if stagger:
        # two submitters, the second starting while the first batches run
        half = len(reqs) // 2
        handles = [None] * len(reqs)

        def sub(lo, hi):
            for i in range(lo, hi):
                s, c = reqs[i]
                handles[i] = server.submit(ids[s], c)
        t1 = threading.Thread(target=sub, args=(0, half))
        t2 = threading.Thread(target=sub, args=(half, len(reqs)))
        t1.start()
        t2.start()
        t1.join()
        t2.join()
    else:
        handles = [server.submit(ids[s], c) for s, c in reqs]
    for h in handles:
        out.append(h.result(timeout_ms=60_000))
    return out


@pytest.mark.parametrize("use_graphs", [True, False])
def test_served_images_equal_alone(world, use_graphs):
    from lumen_b200 import serve
    sc, reqs, refs = world
    with serve.Server(work_budget_bytes=1 << 30, max_views_per_batch=8, use_graphs=use_graphs,
                      autotune=False) as srv:
        res = serve_all(srv, sc, reqs, stagger=True)
        st = srv.stats()
    for i, (r, ref) in enumerate(zip(res, refs)):
        assert r.status == 0
        assert torch.equal(r.image, ref), f"request {i} differs from its standalone render"
        assert r.done_ms >= r.start_ms >= r.submit_ms
    assert st["completed"] == len(reqs) and st["rejected"] == 0
    assert st["batches"] < len(reqs), "no batching happened"
    if use_graphs:
        assert st["graph_launches"] == st["batches"]


@pytest.mark.parametrize("chunk,items", [(128, 16), (512, 8), (256, 8)])
def test_every_launch_variant_gives_the_same_images(world, chunk, items):
    from lumen_b200 import serve
    sc, reqs, refs = world
    with serve.Server(work_budget_bytes=1 << 30, max_views_per_batch=6, autotune=False, composite_chunk=chunk,
                      sort_items=items) as srv:
        res = serve_all(srv, sc, reqs[:12])
    for r, ref in zip(res, refs[:12]):
        assert (r.composite_chunk, r.sort_items) == (chunk, items)
        assert torch.equal(r.image, ref)


def test_autotuner_explores_variants(world):
    from lumen_b200 import serve
    sc, reqs, refs = world
    # one view per batch, one slot: every batch is its own tuner sample
    with serve.Server(work_budget_bytes=1 << 30, max_views_per_batch=1, max_batches_in_flight=1,
                      autotune=True) as srv:
        ids = [srv.add_scene(s) for s in sc]
        seen = set()
        for rep in range(16):
            s, c = reqs[1]
            r = srv.submit(ids[s], c).result(timeout_ms=60_000)
            assert r.status == 0 and torch.equal(r.image, refs[1])
            seen.add((r.composite_chunk, r.sort_items))
    assert len(seen) == 6


def test_instance_overflow_requeues_and_still_matches():
    """Large splats make far more instances than the first estimate; the
    batch that overflows its slot is re-run (split) and every image is
    still exact. The splat size and the budget are chosen from measured
    instance counts so that two views are admitted together (by their
    estimates) but only one fits."""
    from lumen_b200 import render as R
    from lumen_b200 import serve
    n = 4000
    sc = scenes.box_scene(n, seed=50)
    cams = scenes.orbit_cameras(4, 320, 240, radius=8.0)
    est = int(8 * 0.5 * n) + 65536          # the server's first estimate at 240 lines
    chosen = None
    for factor in (8.0, 16.0, 32.0, 64.0):
        big = scenes.Scene(sc.means, (sc.log_scales + np.log(factor)).astype(np.float32), sc.quats,
                           sc.opacity_logits, sc.sh)
        ds = device_scene(big)
        alone = [R.render(*ds.tensors, c, OPT) for c in cams]
        k = [a.n_instances for a in alone]
        max_inst = int(1.2 * max(k))
        if 2 * est <= max_inst < k[0] + k[1]:
            chosen = (ds, alone, k, max_inst)
            break
    assert chosen is not None, "no splat size gives the wanted instance counts"
    ds, alone, k, max_inst = chosen
    refs = [(a.rgb.clamp(0.0, 1.0) * 255.0).to(torch.uint8).cpu() for a in alone]
    budget_per_slot = int(max_inst * 18 / 0.55) + 1
    with serve.Server(work_budget_bytes=2 * budget_per_slot, max_views_per_batch=4, autotune=False) as srv:
        st = srv.stats()
        assert abs(st["max_instances"] - max_inst) <= 2 and st["max_pixels"] >= 2 * 320 * 240
        sid = srv.add_scene(ds)
        hs = [srv.submit(sid, c) for c in cams]
        res = [h.result(timeout_ms=60_000) for h in hs]
        st = srv.stats()
    assert st["requeued_batches"] >= 1 and st["rejected"] == 0
    for r, ref, kv in zip(res, refs, k):
        assert r.status == 0 and torch.equal(r.image, ref)
        assert r.n_instances == kv


def test_request_too_large_for_a_slot_is_rejected():
    from lumen_b200 import serve
    ds = device_scene(scenes.box_scene(1000, seed=51))
    with serve.Server(work_budget_bytes=2 * 40 << 20) as srv:
        sid = srv.add_scene(ds)
        big = ViewCamera.from_fov(8000, 8000, 50.0)
        r = srv.submit(sid, big).result(timeout_ms=60_000)
        ok = srv.submit(sid, ViewCamera.from_fov(64, 48, 50.0)).result(timeout_ms=60_000)
        st = srv.stats()
    assert r.status == -2 and st["rejected"] == 1     # LUMEN_ERROR_OUT_OF_MEMORY
    assert ok.status == 0


def test_frozen_tuning_explores_nothing_and_images_unchanged(world):
    """After a warm-up in which the autotuner explores, freezing it stops
    every exploratory pick (the stats counter stays put) and the served
    images still equal their alone-renders."""
    from lumen_b200 import serve
    sc, reqs, refs = world
    with serve.Server(work_budget_bytes=1 << 30, max_views_per_batch=8, max_batches_in_flight=2,
                      use_graphs=True, autotune=True, options=OPT) as srv:
        serve_all(srv, sc, reqs)
        warm = srv.stats()
        assert warm["explored_batches"] > 0
        srv.freeze_tuning(True)
        ids = list(range(len(sc)))
        res = [srv.submit(ids[s], c) for s, c in reqs]
        out = [h.result(timeout_ms=60_000) for h in res]
        after = srv.stats()
        assert after["explored_batches"] == warm["explored_batches"]
        assert after["batches"] > warm["batches"]
        for r, ref in zip(out, refs):
            assert r.status == 0 and torch.equal(r.image, ref)
        srv.freeze_tuning(False)


def test_batches_hold_at_most_65536_tiles():
    """Admission stops before a batch's tiles pass 65 536 (batch-wide tile
    ids of 16 bits, two tile-sort passes): 1080p views (8160 tiles) go at
    most eight to a batch even when more are queued and max_views_per_batch
    allows more; a view of more tiles than that is rendered alone. Every
    image equals its standalone render."""
    from lumen_b200 import serve
    ds = device_scene(scenes.box_scene(3000, seed=52))
    cams = scenes.orbit_cameras(20, 1920, 1080, radius=9.0)
    wide = ViewCamera.from_fov(4200, 4200, 50.0)          # 263 x 263 = 69 169 tiles
    with serve.Server(work_budget_bytes=4 << 30, max_views_per_batch=64, max_batches_in_flight=1,
                      autotune=False) as srv:
        st = srv.stats()
        assert st["max_tiles"] >= 263 * 263 and st["max_pixels"] >= 4200 * 4200
        sid = srv.add_scene(ds)
        hs = [srv.submit(sid, c) for c in cams]
        res = [h.result(timeout_ms=60_000) for h in hs]
        w = srv.submit(sid, wide).result(timeout_ms=60_000)
    views = [r.batch_views for r in res]
    assert all(r.status == 0 for r in res) and max(views) <= 8 and max(views) >= 2, views
    for i in (0, 7, 19):
        assert torch.equal(res[i].image, alone_u8(ds, cams[i]))
    assert w.status == 0 and w.batch_views == 1
    assert torch.equal(w.image, alone_u8(ds, wide))
