"""Develop request server (lre_server_*): continuous batching under a
device-memory budget.  A request's result must not depend on what else is
in flight: the same request alone and inside a mix of other sizes, CFA
layouts and option sets gives bit-identical output, and matches the plain
per-image path."""
import threading

import numpy as np
import pytest

from libraw_enhanced_b200 import scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lre():
    import libraw_enhanced_b200 as m

    return m


@pytest.fixture(scope="module")
def acc(lre):
    a = lre.CudaAccelerator(0)
    yield a
    a.close()


def _request(lre, i, h, w, bayer=True):
    rng = np.random.default_rng(500 + i)
    if bayer:
        cfa = scenes.random_cfa_name(rng)
        wb = (float(rng.uniform(1.5, 2.5)), 1.0, float(rng.uniform(1.2, 2.0)), 1.0)
        m = scenes.bayer_scene(h, w, 500 + i, cfa=cfa, wb=wb)
        p = lre.develop_params(cfa=cfa, cam_mul=wb)
    else:
        m = scenes.mosaic(scenes.scene_rgb(h, w, 500 + i), scenes.XTRANS_STD, (1.8, 1.0, 1.6, 1.0), 500 + i)
        p = lre.develop_params(cfa=scenes.XTRANS_STD, cam_mul=(1.8, 1.0, 1.6, 1.0))
    p.defringe = int(rng.random() < 0.5)
    p.axial_ca_correction = int(rng.random() < 0.5)
    p.lateral_ca_correction = int(rng.random() < 0.2)
    p.tone_mapping = int(rng.random() < 0.3)
    return m, p


def test_same_result_alone_and_in_mix(lre, acc):
    srv = lre.Server(0, lanes=4)
    try:
        m0, p0 = _request(lre, 0, 384, 512)
        p0.defringe, p0.axial_ca_correction, p0.tone_mapping = 1, 1, 1
        alone, st = srv.wait(srv.submit(m0, p0))
        assert st["total_ms"] >= st["run_ms"] > 0
        assert np.array_equal(alone, acc.develop(m0, p0))
        # a mix of sizes / CFAs / option sets, submitted from two threads,
        # with the same request in the middle
        mix = [_request(lre, i, *hw, bayer=(i % 3 != 2)) for i, hw in
               enumerate([(256, 384), (300, 420), (192, 288), (420, 300), (264, 396), (200, 200)], start=1)]
        tickets = [None] * (len(mix) + 1)

        def submit(idx):
            for k in idx:
                if k == len(mix):
                    tickets[k] = srv.submit(m0, p0)
                else:
                    tickets[k] = srv.submit(*mix[k])

        t1 = threading.Thread(target=submit, args=([0, 2, 4, len(mix)],))
        t2 = threading.Thread(target=submit, args=([1, 3, 5],))
        t1.start(), t2.start(), t1.join(), t2.join()
        outs = [srv.wait(t) for t in tickets]
        assert np.array_equal(outs[-1][0], alone)
        for (m, p), (o, s) in zip(mix, outs[:-1]):
            assert np.array_equal(o, acc.develop(m, p)), s
        lanes = {s["lane"] for _, s in outs}
        assert len(lanes) > 1  # requests ran on several lanes
        in_use, peak = srv.memory()
        assert peak > 0 and in_use <= peak
    finally:
        srv.close()


def test_budget_admission(lre, acc):
    m, p = _request(lre, 9, 256, 384)
    p.defringe, p.axial_ca_correction = 1, 1
    # room for one request's buffers at a time: everything still completes,
    # one after another, and the resident peak stays inside the budget
    probe = lre.Server(0, lanes=1)
    try:
        _, st = probe.wait(probe.submit(m, p))
        need = st["device_bytes"]
    finally:
        probe.close()
    budget = int(need * 1.5)
    srv = lre.Server(0, lanes=3, budget_bytes=budget)
    try:
        ts = [srv.submit(m, p) for _ in range(4)]
        outs = [srv.wait(t) for t in ts]
        ref = acc.develop(m, p)
        for o, s in outs:
            assert np.array_equal(o, ref)
        _, peak = srv.memory()
        assert 0 < peak <= budget
    finally:
        srv.close()
    # a request larger than the whole budget is refused at submit
    srv = lre.Server(0, lanes=2, budget_bytes=1 << 20)
    try:
        with pytest.raises(lre.LibRawError) as ei:
            srv.submit(m, p)
        assert ei.value.status == 7
    finally:
        srv.close()


def test_wait_timeout_and_invalid(lre):
    srv = lre.Server(0, lanes=1)
    try:
        with pytest.raises(lre.LibRawError):
            srv.submit(np.zeros((8, 8), np.float32), lre.develop_params())
        m, p = _request(lre, 3, 512, 768)
        p.defringe = 1
        t = srv.submit(m, p)
        out, st = srv.wait(t, timeout_ms=60000)
        assert out.shape == (512, 768, 3)
    finally:
        srv.close()


def test_decode_callbacks_overlap_device_work(lre, acc):
    """lre_server_submit_decode: a host decode step (here a stand-in for
    LibRaw's unpack: a 14-bit integer raw plane scaled to float, with a
    50 ms delay) runs on the server's decode threads while the lanes develop
    earlier requests.  Results equal the plain path's bit for bit; two
    decode threads finish six requests in well under the serial time; an
    error in one decode fails that request only."""
    import time

    srv = lre.Server(0, lanes=2, decode_threads=2)
    try:
        raws, params, expect = [], [], []
        for i in range(6):
            m, p = _request(lre, 20 + i, 256, 384)
            raw = np.clip(np.rint(m * 16383.0), 0, 16383).astype(np.uint16)
            raws.append(raw)
            params.append(p)
            expect.append(acc.develop(raw.astype(np.float32) / np.float32(16383.0), p))

        def decoder(raw):
            def fill(mosaic):
                time.sleep(0.05)
                np.divide(raw.astype(np.float32), np.float32(16383.0), out=mosaic)
            return fill

        t0 = time.perf_counter()
        tickets = [srv.submit_decode(r.shape, p, decoder(r)) for r, p in zip(raws, params)]
        results = [srv.wait(t) for t in tickets]
        wall_ms = (time.perf_counter() - t0) * 1e3
        serial_ms = 0.0
        for (out, st), e in zip(results, expect):
            assert np.array_equal(out, e)
            assert st["decode_ms"] >= 45.0
            serial_ms += st["decode_ms"] + st["run_ms"]
        assert wall_ms < 0.75 * serial_ms, (wall_ms, serial_ms)

        def broken(mosaic):
            raise RuntimeError("corrupt raw file")

        bad = srv.submit_decode((64, 96), params[0], broken)
        good = srv.submit_decode(raws[0].shape, params[0], decoder(raws[0]))
        with pytest.raises(RuntimeError, match="corrupt raw file"):
            srv.wait(bad)
        out, _ = srv.wait(good)
        assert np.array_equal(out, expect[0])
    finally:
        srv.close()
