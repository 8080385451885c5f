"""GPU tests of the serving form (at_server_*) and of batches of uneven
frames: each frame's result is the same alone and in the mix."""
import time

import numpy as np
import pytest

import apriltags_fast_b200 as AT
from apriltags_fast_b200 import synth
from oracle import oracle as O
from tests import helpers as H

pytestmark = pytest.mark.gpu


def _alone(det, frames):
    out = []
    for f in frames:
        d = det.detect_batch([f], as_arrays=True)[0]
        out.append((d.tobytes(), det.last_batch_nquads[0]))
    return out


def _drain(srv, n, timeout_s=60.0):
    got = []
    t0 = time.time()
    while len(got) < n and time.time() - t0 < timeout_s:
        got += srv.poll(64, wait_ms=50)
    return got


def test_server_results_equal_alone():
    frames = synth.serve_mix(6, 11) + H.golden_images()
    det = AT.Detector(["tag36h11"], 2)
    alone = _alone(det, frames)
    srv = AT.Server(det, workers=2, max_batch=4)
    try:
        tickets = []
        for rep in range(3):
            for i, f in enumerate(frames):
                t = srv.submit(f, user=i)
                assert t > 0
                tickets.append(t)
        res = _drain(srv, len(tickets))
        assert len(res) == len(tickets)
        assert sorted(r["ticket"] for r in res) == sorted(tickets)
        assert any(r["batch_frames"] > 1 for r in res)  # frames were batched together
        for r in res:
            assert r["status"] == 0
            assert (r["detections"].tobytes(), r["nquads"]) == alone[r["user"]]
            assert r["t_submit"] <= r["t_start"] <= r["t_done"]
        st = srv.stats()
        assert st["completed"] == len(tickets) and st["rejected"] == 0 and st["pending"] == 0
    finally:
        srv.close()


def test_server_single_request_equals_at_detect():
    img = H.golden_images()[0]
    det = AT.Detector(["tag36h11"], 2)
    ref = det.detect(img)
    srv = AT.Server(det, workers=1, max_batch=8)
    try:
        assert srv.submit(img, user=7) > 0
        (r,) = _drain(srv, 1)
        assert r["user"] == 7 and r["batch_frames"] == 1
        assert len(r["detections"]) == len(ref)
        for a, b in zip(r["detections"], ref):
            assert int(a["id"]) == b.id and float(a["decision_margin"]) == b.decision_margin
            assert tuple(a["H"]) == b.H
    finally:
        srv.close()


def test_server_admission_by_memory_budget():
    """A frame that alone needs more than a worker's share of the budget is
    rejected; smaller frames are admitted and finish."""
    det = AT.Detector(["tag36h11"], 2)
    srv = AT.Server(det, workers=2, max_batch=4, memory_budget=64 << 20)
    try:
        big = np.zeros((2160, 3840), np.uint8)
        small = H.golden_images()[0]
        assert srv.submit(big) == 0
        assert srv.submit(small) > 0
        res = _drain(srv, 1)
        assert len(res) == 1 and res[0]["status"] == 0
        st = srv.stats()
        assert st["rejected"] == 1 and st["admitted"] == 1
    finally:
        srv.close()


def test_uneven_batch_with_family_sets_equals_single():
    """Frames of four sizes with per-frame family sets in one batch: each
    frame's detections equal the same frame run alone."""
    frames, fams = synth.uneven_batch(8, 5)
    det = AT.Detector(["tag36h11", "tag25h9"], 2)
    masks = [1 if f == "tag36h11" else 2 for f in fams]
    batch = det.detect_batch(frames, family_masks=masks, as_arrays=True)
    nq = list(det.last_batch_nquads)
    for i, f in enumerate(frames):
        one = det.detect_batch([f], family_masks=[masks[i]], as_arrays=True)[0]
        assert one.tobytes() == batch[i].tobytes()
        assert det.last_batch_nquads[0] == nq[i]
        assert all(int(x["family"]) == (0 if masks[i] == 1 else 1) for x in one)


def test_uneven_batch_of_64_equals_reference_per_frame():
    """The batched workload: 64 frames of sizes drawn from 640x480 to
    3840x2160, each with 0-40 tags of tag36h11 or tag25h9 (codes drawn with
    replacement) and its own family set, in one batch. Each frame's
    detections and quad count equal the reference's own (oracle/_ref, one
    thread) run on that frame alone with that frame's family, in its order;
    the family index is the detector's (0 or 1)."""
    if O.ref_lib() is None:
        pytest.skip("oracle/_ref not built")
    frames, fams = synth.uneven_batch(64, 5)
    det = AT.Detector(["tag36h11", "tag25h9"], 2)
    masks = [1 if f == "tag36h11" else 2 for f in fams]
    batch = det.detect_batch(frames, family_masks=masks)
    nq = list(det.last_batch_nquads)
    sizes = set()
    for i, f in enumerate(frames):
        ref, ref_nq = O.ref_detect(f, [fams[i]], [2])
        got = [d.key() for d in batch[i]]
        fi = 0 if fams[i] == "tag36h11" else 1
        assert all(g[0] == fi for g in got), i
        assert [g[1:] for g in got] == [r[1:] for r in ref], i
        assert nq[i] == ref_nq, i
        sizes.add(f.shape)
    assert len(sizes) == 4


def test_batch_split_equals_one_pipeline():
    """A batch spread over 2-4 pipelines (helper detectors on their own
    threads) gives the same detections and quad counts, frame by frame, as
    one pipeline."""
    frames, fams = synth.uneven_batch(40, 9)
    det = AT.Detector(["tag36h11", "tag25h9"], 2)
    masks = [1 if f == "tag36h11" else 2 for f in fams]
    det.set_batch_split(1)
    ref = [d.tobytes() for d in det.detect_batch(frames, family_masks=masks, as_arrays=True)]
    ref_nq = list(det.last_batch_nquads)
    for p in (2, 3, 4, 2):
        det.set_batch_split(p)
        got = det.detect_batch(frames, family_masks=masks, as_arrays=True)
        assert [d.tobytes() for d in got] == ref
        assert list(det.last_batch_nquads) == ref_nq
    with pytest.raises(ValueError):
        det.set_batch_split(5)


def test_shutdown_with_batch_pipelines_then_detect_again():
    """at_shutdown releases the arenas of the detector and of its batch
    helpers; the next batch allocates them again and gives the same bytes."""
    frames, _ = synth.uneven_batch(20, 4)
    det = AT.Detector(["tag36h11"], 2)
    first = [d.tobytes() for d in det.detect_batch(frames, as_arrays=True)]
    det.shutdown()
    again = [d.tobytes() for d in det.detect_batch(frames, as_arrays=True)]
    assert again == first


def test_server_cancel_queued_requests():
    """Requests cancelled while still queued come back with status
    SERVER_CANCELLED and no detections; the others complete unchanged."""
    det = AT.Detector(["tag36h11"], 2)
    frames = synth.serve_mix(4, 21) + H.golden_images()
    alone = _alone(det, frames)
    big = synth.make_frame(synth.CONFIGS["serve_2160p"], 5)[0]
    srv = AT.Server(det, workers=1, max_batch=1)
    try:
        first = srv.submit(big, user=99)  # keeps the one worker busy
        tickets = [(srv.submit(f, user=i), i) for i, f in enumerate(frames) for _ in range(2)]
        cancelled = {t for t, _ in tickets[1::2] if srv.cancel(t)}
        assert len(cancelled) >= len(tickets) // 2 - 1
        res = _drain(srv, len(tickets) + 1)
        assert len(res) == len(tickets) + 1
        for r in res:
            if r["ticket"] in cancelled:
                assert r["status"] == AT.SERVER_CANCELLED and len(r["detections"]) == 0
            elif r["user"] != 99:
                assert r["status"] == 0
                assert (r["detections"].tobytes(), r["nquads"]) == alone[r["user"]]
        st = srv.stats()
        assert st["cancelled"] == len(cancelled) and st["pending"] == 0
    finally:
        srv.close()


def test_server_rejects_when_queued_bytes_exceed_budget():
    """A burst bigger than the budget: the frames whose queued device bytes
    would pass the budget are turned away; the admitted ones finish."""
    det = AT.Detector(["tag36h11"], 2)
    img = H.golden_images()[0]
    srv = AT.Server(det, workers=1, max_batch=2, memory_budget=80 << 20)
    try:
        tickets = [srv.submit(img, user=i) for i in range(40)]
        admitted = [t for t in tickets if t > 0]
        assert 0 < len(admitted) < len(tickets)
        res = _drain(srv, len(admitted))
        assert len(res) == len(admitted) and all(r["status"] == 0 for r in res)
        st = srv.stats()
        assert st["rejected"] == len(tickets) - len(admitted)
    finally:
        srv.close()


def test_server_over_a_device_list():
    """Workers dealt out over a list of GPUs (one detector replica each; this
    box has one GPU, listed for both workers): each worker reports its GPU
    and every result equals the frame alone, from host frames and from
    device frames. A mask that names no GPU of this machine is refused."""
    import torch

    frames = synth.serve_mix(4, 5)
    det = AT.Detector(["tag36h11"], 2)
    alone = _alone(det, frames)
    dev = [torch.from_numpy(np.ascontiguousarray(f)).cuda() for f in frames]
    srv = AT.Server(det, workers=2, max_batch=4, devices=[0])
    try:
        assert [srv.worker_device(w) for w in range(3)] == [0, 0, -1]
        tickets = [srv.submit(f, user=i) for i, f in enumerate(frames)]
        tickets += [srv.submit(f, user=i) for i, f in enumerate(dev)]
        assert all(t > 0 for t in tickets)
        res = _drain(srv, len(tickets))
        assert sorted(r["ticket"] for r in res) == sorted(tickets)
        for r in res:
            assert r["status"] == 0 and srv.worker_device(r["worker"]) == 0
            assert (r["detections"].tobytes(), r["nquads"]) == alone[r["user"]]
    finally:
        srv.close()
    with pytest.raises(RuntimeError):
        AT.Server(det, workers=1, devices=[31])
