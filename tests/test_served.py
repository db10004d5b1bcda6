"""Batch and served entry points (culs_rw_st_batch, culs_submit / culs_poll /
culs_wait / culs_fetch): every result equals the oracle's `rw; st` of the
same graph, exactly, whichever batch a graph or job ends up in."""
import numpy as np
import pytest

import culs_b200 as C
from util import oracle_rw_st, same_graph

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = C.Context()
    yield c
    c.close()


def graphs():
    return [C.gen_multiplier(8), C.gen_layered(21, 32, 16, 3000, 30, 4, 0.0, True), C.gen_multiplier(12),
            C.gen_layered(22, 64, 32, 9000, 60, 3, 0.2, False), C.gen_layered(23, 16, 8, 700, 20, 4, 0.0, True)]


def test_rw_st_batch_over_handles(ctx):
    gs = graphs()
    hs = [ctx.upload(gs[0]), ctx.upload_batch(gs[1:3]), ctx.upload(gs[3]), ctx.upload_batch(gs[4:])]
    ctx.rw_st_batch(hs)
    got = [hs[0].download()] + hs[1].download_all() + [hs[2].download()] + hs[3].download_all()
    assert len(got) == len(gs)
    for i, (a, g) in enumerate(zip(got, gs)):
        ref = oracle_rw_st(g).graph()
        assert same_graph(a, ref), i
        assert a.nLevels == ref.nLevels, i


def test_rw_st_batch_rejects_repeated_handle(ctx):
    h = ctx.upload(C.gen_multiplier(6))
    with pytest.raises(C.CulsError) as e:
        ctx.rw_st_batch([h, h])
    assert e.value.code == -1


def test_served_jobs_match_oracle(ctx):
    gs = graphs()
    # a small admission budget and batch cap, so the jobs run as several batches
    ctx.serve_start(admit_bytes=C.SERVE_BYTES_PER_OBJ * 12000, max_batch=3)
    try:
        jobs = [(ctx.submit(g, zeros=(i == 2)), g, i == 2) for i, g in enumerate(gs * 2)]
        for job, g, zeros in jobs:
            assert ctx.wait(job, 60000)
            out, lat = ctx.fetch(job)
            ref = oracle_rw_st(g, zeros=zeros).graph()
            assert same_graph(out, ref), job
            assert out.nLevels == ref.nLevels
            assert lat >= 0.0
            with pytest.raises(C.CulsError) as e:  # a fetched job is forgotten
                ctx.poll(job)
            assert e.value.code == C.CULS_E_NOTFOUND
        with pytest.raises(C.CulsError) as e:
            ctx.poll(10 ** 9)
        assert e.value.code == C.CULS_E_NOTFOUND
    finally:
        ctx.serve_stop()


def test_served_workers_match_oracle(ctx):
    # three workers, each with an engine of its own, take their shares of a burst
    gs = graphs()
    ctx.serve_start(workers=3)
    try:
        jobs = [(ctx.submit(g), g) for g in gs * 3]
        for job, g in jobs:
            assert ctx.wait(job, 60000)
            out, _ = ctx.fetch(job)
            ref = oracle_rw_st(g).graph()
            assert same_graph(out, ref), job
            assert out.nLevels == ref.nLevels
    finally:
        ctx.serve_stop()
    # direct calls on the context still work after the server stopped
    h = ctx.upload(gs[0])
    ctx.rw_st_batch([h])
    assert same_graph(h.download(), oracle_rw_st(gs[0]).graph())


def test_served_aiger_jobs_match_oracle(ctx, tmp_path):
    """Jobs given as binary AIGER bytes, mixed with array jobs: decoded and
    encoded on the device in batches of their own kind; a file whose header
    is fine but whose AND section does not decode fails its own job only."""
    gs = graphs()
    files = []
    for i, g in enumerate(gs):
        p = tmp_path / f"j{i}.aig"
        C.write_aiger(p, g)
        files.append(p.read_bytes())
    bad = b"aig 3 2 0 1 1\n6\n\x00\x02c\n"  # delta 0: the fanin does not precede its node
    ctx.serve_start(workers=2)
    try:
        jobs = []
        for i, (g, f) in enumerate(zip(gs * 2, files * 2)):
            jobs.append(("aig", ctx.submit_aiger(f, zeros=(i == 1)), g, i == 1))
            if i == 2:
                jobs.append(("bad", ctx.submit_aiger(bad), None, False))
            jobs.append(("arr", ctx.submit(g), g, False))
        with pytest.raises(C.CulsError) as e:  # a header the host reader refuses
            ctx.submit_aiger(b"aag 1 1 0 1 0\n2\n")
        assert e.value.code == C.CULS_E_IO
        for kind, job, g, zeros in jobs:
            if kind == "bad":
                with pytest.raises(C.CulsError) as e:
                    ctx.wait(job, 60000)
                assert e.value.code == C.CULS_E_IO
                continue
            assert ctx.wait(job, 60000)
            ref = oracle_rw_st(g, zeros=zeros).graph()
            if kind == "aig":
                data, lat = ctx.fetch_aiger(job)
                p = tmp_path / "out.aig"
                p.write_bytes(data)
                out = C.read_aiger(p)
            else:
                out, lat = ctx.fetch(job)
            assert same_graph(out, ref), (kind, job)
            assert lat >= 0.0
    finally:
        ctx.serve_stop()


def test_served_job_error_is_reported():
    small = C.Context(hbm_budget=1 << 20)
    small.serve_start()
    try:
        job = small.submit(C.gen_multiplier(16))
        with pytest.raises(C.CulsError) as e:  # wait returns the job's outcome
            small.wait(job, 60000)
        assert e.value.code == -3  # CULS_E_BUDGET, carried to the job
        with pytest.raises(C.CulsError) as e:
            small.fetch(job)
        assert e.value.code == -3
    finally:
        small.serve_stop()
        small.close()


def test_cancel_queued_job(ctx):
    # one worker taking one job per batch: the second job waits in the queue
    # while the first (a 300k-AND graph) runs
    big, small = C.gen_layered(31, 256, 64, 300000, 200, 4, 0.0, True), C.gen_multiplier(8)
    ctx.serve_start(max_batch=1, workers=1)
    try:
        j1 = ctx.submit(big)
        j2 = ctx.submit(small)
        ctx.cancel(j2)
        with pytest.raises(C.CulsError) as e:  # finished at once, with its code
            ctx.wait(j2, 0)
        assert e.value.code == C.CULS_E_CANCELLED
        with pytest.raises(C.CulsError) as e:
            ctx.poll(j2)
        assert e.value.code == C.CULS_E_CANCELLED
        with pytest.raises(C.CulsError) as e:  # fetching reports the code and forgets the job
            ctx.fetch(j2)
        assert e.value.code == C.CULS_E_CANCELLED
        with pytest.raises(C.CulsError) as e:
            ctx.poll(j2)
        assert e.value.code == C.CULS_E_NOTFOUND
        with pytest.raises(C.CulsError) as e:
            ctx.cancel(10 ** 9)
        assert e.value.code == C.CULS_E_NOTFOUND
        assert ctx.wait(j1, 120000)
        with pytest.raises(C.CulsError) as e:  # a finished job is not cancelled
            ctx.cancel(j1)
        assert e.value.code == C.CULS_E_INVALID
        out, _ = ctx.fetch(j1)
        assert same_graph(out, oracle_rw_st(big).graph())
    finally:
        ctx.serve_stop()


def test_bad_job_fails_alone(ctx):
    """A malformed graph (a fanin that is not below its node) batched with
    valid ones fails with CULS_E_INVALID; the others still match the oracle."""
    big = C.gen_layered(32, 256, 64, 300000, 200, 4, 0.0, True)
    good = [C.gen_multiplier(8), C.gen_layered(33, 32, 16, 3000, 30, 4, 0.0, True)]
    m = C.gen_multiplier(6)
    f0 = np.array(m.fanin0, copy=True)
    f0[-1] = 2 * (len(f0) - 1)  # the last AND node as its own fanin
    bad = C.Aig(m.nPIs, f0, np.asarray(m.fanin1), np.asarray(m.outs))
    ctx.serve_start(workers=1)
    try:
        j0 = ctx.submit(big)  # runs while the next three queue up as one batch
        js = [ctx.submit(good[0]), ctx.submit(bad), ctx.submit(good[1])]
        for j in [j0] + js:
            try:
                ctx.wait(j, 120000)
            except C.CulsError:
                pass
        with pytest.raises(C.CulsError) as e:
            ctx.fetch(js[1])
        assert e.value.code == C.CULS_E_INVALID
        for j, g in [(j0, big), (js[0], good[0]), (js[2], good[1])]:
            out, _ = ctx.fetch(j)
            assert same_graph(out, oracle_rw_st(g).graph())
    finally:
        ctx.serve_stop()
