"""The live ingestion ring (reference ptyrs/src/live/ring.rs, its single-store tests at
ring.rs:1240-1410): frames land in sequence order once their positions are in; a frame
without a position is dropped after the wait, or at once when a worker needs its slot; one
with an invalid position is dropped without waiting; a full ring holds a frame whose position
comes within the wait. The device store then holds the same counts `GpuPtycho` converts: a
state made from the ring runs rPIE to the same arrays as one made by `GpuPtycho` from the
landed frames."""
import threading
import time

import numpy as np
import pytest

from ptyrs_b200 import GpuPtycho, PtybError, Scan, sim
from ptyrs_b200.live import LiveRing
from scenarios import far_field

pytestmark = pytest.mark.gpu

HOUR = 3600.0


@pytest.fixture(scope="module")
def scan():
    s = far_field(64, 2, 48, 192, masked=True)
    s["u16"] = np.where(s["counts"] < 0, 65535, s["counts"]).astype(np.uint16)
    return s


def ring(n=64, **kw):
    return LiveRing(n, sim.WAVELENGTH, sim.DISTANCE, sim.DETECTOR_PIXEL, **kw)


def landed(r):
    return list(r.landed()[0])


def test_frames_land_in_order_and_run_as_a_created_scan(scan):
    nframe = len(scan["u16"])
    # a ring that holds every frame: half the positions come before their frames, the rest
    # after, in reverse order, and no worker needs a slot meanwhile
    with ring(slots=64, capacity=64, batch=5) as r:
        for f in range(0, nframe, 2):
            r.position(1000 + f, scan["y"][f], scan["x"][f])
        for f in range(nframe):
            r.put(1000 + f, scan["u16"][f])
        for f in reversed(range(1, nframe, 2)):
            r.position(1000 + f, scan["y"][f], scan["x"][f])
        r.flush(10.0)
        st = r.stats()
        assert (st["committed"], st["landed"], st["ready"]) == (nframe, nframe, nframe)
        assert st["dropped_no_position"] + st["dropped_invalid"] + st["dropped_full"] == 0
        uids, y, x = r.landed()
        assert list(uids) == [1000 + f for f in range(nframe)]
        np.testing.assert_array_equal(y, scan["y"])
        np.testing.assert_array_equal(x, scan["x"])
        with r.gpu_ptycho(scan["object"], scan["probe"]) as g:
            ref = GpuPtycho(Scan(scan["u16"], scan["y"], scan["x"], sim.WAVELENGTH, sim.DISTANCE,
                                 sim.DETECTOR_PIXEL), scan["object"], scan["probe"])
            assert g.llk() == ref.llk()
            for h in (g, ref):
                h.rpie(2, batch_size=16, seed=3)
            np.testing.assert_array_equal(g.object(), ref.object())
            np.testing.assert_array_equal(g.probe(), ref.probe())
            ref.close()


def test_float_counts_land_and_a_non_finite_frame_is_refused(scan):
    c = scan["counts"][:6].copy()
    with ring(counts="f32", slots=4, capacity=16) as r:
        for f in range(6):
            r.position(f, scan["y"][f], scan["x"][f])
            r.put(f, c[f])
        r.flush(10.0)
        with r.gpu_ptycho(scan["object"], scan["probe"]) as g:
            ref = GpuPtycho(Scan(c, scan["y"][:6], scan["x"][:6], sim.WAVELENGTH, sim.DISTANCE,
                                 sim.DETECTOR_PIXEL), scan["object"], scan["probe"])
            assert g.llk() == ref.llk()
            ref.close()
        bad = c[0].copy()
        bad[10, 10] = np.nan
        r.position(6, scan["y"][6], scan["x"][6])
        r.put(6, bad)
        r.flush(10.0)
        with pytest.raises(PtybError, match="finite"):
            r.gpu_ptycho(scan["object"], scan["probe"])


def test_a_frame_without_a_position_is_dropped_after_the_wait(scan):
    with ring(slots=16, capacity=64, pos_wait_s=0.002) as r:
        for f in range(10):
            if f != 4:
                r.position(f, scan["y"][f], scan["x"][f])
            r.put(f, scan["u16"][f])
        r.flush(10.0)
        st = r.stats()
        assert landed(r) == [0, 1, 2, 3, 5, 6, 7, 8, 9]
        assert (st["dropped_no_position"], st["dropped_crowded"], st["stalls"]) == (1, 0, 0)


def test_a_frame_with_an_invalid_position_is_dropped_at_once(scan):
    with ring(slots=8, capacity=64, pos_wait_s=HOUR) as r:
        r.position(3, np.nan, 0.0)
        for f in range(8):
            if f != 3:
                r.position(f, scan["y"][f], scan["x"][f])
            r.put(f, scan["u16"][f])
        t0 = time.perf_counter()
        r.flush(10.0)
        assert time.perf_counter() - t0 < 5.0
        st = r.stats()
        assert landed(r) == [0, 1, 2, 4, 5, 6, 7]
        assert (st["dropped_invalid"], st["dropped_no_position"]) == (1, 0)


def test_an_invalid_position_ends_its_frames_wait(scan):
    with ring(slots=8, capacity=64, pos_wait_s=HOUR) as r:
        for f in range(6):
            if f:
                r.position(f, scan["y"][f], scan["x"][f])
            r.put(f, scan["u16"][f])
        time.sleep(0.05)
        st = r.stats()
        assert st["landed"] == 0, "a frame landed before frame 0"
        assert st["pos_waits"] == 1
        r.position(0, 0.0, 2e10)
        r.flush(10.0)
        assert landed(r) == [1, 2, 3, 4, 5]
        assert (r.stats()["dropped_invalid"], r.stats()["dropped_no_position"]) == (1, 0)


def test_a_position_within_the_wait_lands_its_frame_behind_a_full_ring(scan):
    with ring(slots=4, capacity=64, pos_wait_s=HOUR) as r:
        for f in range(4):
            if f:
                r.position(f, scan["y"][f], scan["x"][f])
            r.put(f, scan["u16"][f])
        time.sleep(0.05)
        assert r.stats()["landed"] == 0, "a frame landed before frame 0"
        r.position(0, scan["y"][0], scan["x"][0])
        r.flush(10.0)
        st = r.stats()
        assert landed(r) == [0, 1, 2, 3]
        assert (st["dropped_no_position"], st["stalls"]) == (0, 0)


def test_a_frame_without_a_position_is_dropped_once_a_worker_needs_its_slot(scan):
    # single frames and a run longer than the ring lack positions; the ring wraps many times
    missing = {5, 11, 17, 20, 21, 22, 23, 24, 25}
    with ring(slots=4, capacity=64, pos_wait_s=HOUR) as r:
        for f in range(40):
            if f not in missing:
                r.position(f, scan["y"][f], scan["x"][f])
        for f in range(40):
            r.put(f, scan["u16"][f])
        r.flush(10.0)
        st = r.stats()
        assert landed(r) == [f for f in range(40) if f not in missing]
        assert (st["dropped_no_position"], st["dropped_crowded"]) == (len(missing), len(missing))


def test_frames_past_the_store_are_dropped(scan):
    with ring(slots=4, capacity=5) as r:
        for f in range(8):
            r.position(f, scan["y"][f], scan["x"][f])
            r.put(f, scan["u16"][f])
        r.flush(10.0)
        st = r.stats()
        assert (st["landed"], st["dropped_full"]) == (5, 3)
        with r.gpu_ptycho(scan["object"], scan["probe"]) as g:
            assert np.isfinite(g.llk()["poisson"])


def test_workers_on_threads_land_every_frame(scan):
    """Four workers commit frames in their own orders through a ring of six slots while
    positions come from another thread: every frame lands once or is dropped for a position
    that came after a worker needed its slot, and the state over the landing order is the
    created scan's over the same order."""
    nframe = len(scan["u16"])
    order = np.random.default_rng(5).permutation(nframe)
    with ring(slots=6, capacity=64, batch=4, pos_wait_s=HOUR) as r:
        def worker(k):
            for f in order[k::4]:
                r.put(int(f), scan["u16"][f])

        def positions():
            for f in order[::-1]:
                r.position(int(f), scan["y"][f], scan["x"][f])
                time.sleep(0.0002)

        threads = [threading.Thread(target=worker, args=(k,)) for k in range(4)]
        threads.append(threading.Thread(target=positions))
        for t in threads:
            t.start()
        for t in threads:
            t.join(60.0)
        r.flush(20.0)
        uids = np.array(landed(r))
        st = r.stats()
        assert len(set(uids)) == len(uids) > 0
        assert st["committed"] == nframe
        assert st["landed"] + st["dropped_no_position"] == nframe
        assert st["dropped_no_position"] == st["dropped_crowded"]
        with r.gpu_ptycho(scan["object"], scan["probe"]) as g:
            ref = GpuPtycho(Scan(scan["u16"][uids], scan["y"][uids], scan["x"][uids],
                                 sim.WAVELENGTH, sim.DISTANCE, sim.DETECTOR_PIXEL),
                            scan["object"], scan["probe"])
            for h in (g, ref):
                h.rpie(1, batch_size=16, seed=3)
            np.testing.assert_array_equal(g.object(), ref.object())
            ref.close()
