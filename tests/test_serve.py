"""Serving loop (zfpb_server_*): requests admitted by a device-memory budget
and coded in continuously formed batches, each result the same as the
single-array device call gives for that request alone."""

import random
import threading
import time

import numpy as np
import pytest

from tests import zfpb
from tests.test_batch import mixed_jobs

pytestmark = pytest.mark.gpu
Z = zfpb.load()


def prepare(jobs):
    """Per request: input field, stream buffer, the stream and decode that the
    single-array calls give (the expected results)."""
    import torch

    reqs = []
    for x, cfg in jobs:
        cap = Z.maximum_size(x.shape, Z._np_dtype(x.dtype), cfg)
        ref_stream = torch.zeros((cap + 7) // 8, dtype=torch.int64, device="cuda")
        n = Z.compress_device(x, cfg, out=ref_stream)
        ref_out = torch.zeros_like(x)
        Z.decompress_device(ref_stream, n, ref_out, cfg)
        reqs.append(dict(x=x, cfg=cfg, cap=cap, n=n, ref_stream=ref_stream, ref_out=ref_out))
    return reqs


def run_mix(server, reqs, seed, spread_s=0.05):
    """Submit a compress and a decompress per request from another thread at
    random times; return the results by tag."""
    import torch

    rnd = random.Random(seed)
    subs = []
    for i, r in enumerate(reqs):
        cs = torch.zeros_like(r["ref_stream"])
        subs.append((2 * i, Z.batch_items([r["x"]], [r["cfg"]], [cs])[0], False, ("c", i, cs)))
        out = torch.full_like(r["x"], 3)
        subs.append((2 * i + 1, Z.batch_items([out], [r["cfg"]], [r["ref_stream"]], nbytes=[r["n"]])[0], True,
                     ("d", i, out)))
    rnd.shuffle(subs)
    when = sorted(rnd.uniform(0, spread_s) for _ in subs)
    torch.cuda.synchronize()

    def client():
        t0 = time.perf_counter()
        for (tag, item, dec, _), t in zip(subs, when):
            while time.perf_counter() - t0 < t:
                pass
            assert server.submit(item, dec, tag)

    th = threading.Thread(target=client)
    th.start()
    results = {}
    deadline = time.time() + 120
    while len(results) < len(subs) and time.time() < deadline:
        for tag, res, st, q, lat in server.poll(64, wait_ms=50):
            results[tag] = (res, st, q, lat)
    th.join()
    return subs, results


def check(reqs, subs, results):
    import torch

    for tag, _, dec, (kind, i, buf) in subs:
        res, st, q, lat = results[tag]
        r = reqs[i]
        assert st == 0 and res == r["n"], (tag, kind, st, res, r["n"])
        assert q >= 0 and lat >= q
        if kind == "c":
            assert torch.equal(buf[: res // 8], r["ref_stream"][: res // 8]), tag
        else:
            assert torch.equal(buf.view(torch.uint8), r["ref_out"].view(torch.uint8)), tag


def test_results_in_the_mix_equal_results_alone():
    reqs = prepare(mixed_jobs(7, n=30))
    server = Z.Server(4 << 30, lanes=2)
    try:
        subs, results = run_mix(server, reqs, seed=1)
        assert len(results) == len(subs)
        check(reqs, subs, results)
        assert server.outstanding() == 0
    finally:
        server.close()


def test_small_budget_admits_in_order_and_rejects_oversized():
    import torch

    reqs = prepare(mixed_jobs(8, n=12))
    biggest = max(r["x"].numel() * r["x"].element_size() + r["cap"] for r in reqs)
    # A budget barely above the largest request: requests run a few at a time.
    server = Z.Server(2 * biggest + (64 << 20), lanes=2, max_batch=3)
    try:
        subs, results = run_mix(server, reqs, seed=2, spread_s=0.0)
        check(reqs, subs, results)
        huge = torch.zeros((1 << 14, 1 << 13), dtype=torch.float32, device="cuda")
        cfg = Z.ZfpConfig.fixed_precision(30)
        sb = torch.zeros(1, dtype=torch.int64, device="cuda")
        item = Z.batch_items([huge], [cfg], [sb])[0]
        item.stream_bytes = 8 << 30
        assert not server.submit(item, False, 999)
        assert Z.lib().zfpb_last_error() == 6
    finally:
        server.close()
