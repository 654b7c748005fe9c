"""CPU checks of the stream staging plan (hcgrid_b200/streams.py): windows
respect the staging budget and keep stream order, oversized requests get a
window of their own, and a field's last use is its last request."""
from hcgrid_b200 import streams, synth


def test_windows_fit_budget_and_keep_order():
    reqs = synth.config5_requests(njobs=400, seed=3, reuse=0.3, max_grid=2048)
    budget = 24 << 30
    wins = streams.plan_windows(reqs, budget)
    flat = [r["request"] for w in wins for r in w]
    assert flat == [r["request"] for r in reqs]
    for w in wins:
        total = sum(streams.footprint(r["shape"]) for r in w)
        assert total <= budget or len(w) == 1


def test_last_use_and_work():
    reqs = [dict(request=i, field=f, shape=dict(n=10, nchan=c, grid=8), spectra_seed=0)
            for i, (f, c) in enumerate([(0, 1), (1, 64), (0, 2), (2, 4), (1, 8)])]
    assert streams.last_use(reqs) == {0: 2, 1: 4, 2: 3}
    assert [streams.request_work(r) for r in reqs] == [10, 640, 20, 40, 80]


def test_config5_stream_is_uncapped():
    """The full served stream keeps config-4's largest shapes (no redraws)."""
    reqs = synth.config5_requests(njobs=2000, seed=3, reuse=0.3, max_grid=2048)
    assert len(reqs) == 2000
    assert max(r["shape"]["n"] * r["shape"]["nchan"] for r in reqs) > 1 << 31
    assert max(r["shape"]["grid"] for r in reqs) == 2048


def test_fills_gpu_matches_the_server_rule():
    """Large jobs: 2^20 pixels, or one 16x8-pixel x 256-channel item per SM."""
    sh = lambda g, c: {"grid": g, "nchan": c}
    assert streams.fills_gpu(sh(1024, 1)) and streams.fills_gpu(sh(2048, 64))
    assert not streams.fills_gpu(sh(512, 1))           # single channel below 2^20 pixels
    assert streams.fills_gpu(sh(256, 64))              # 512 tiles
    assert not streams.fills_gpu(sh(128, 256))         # 128 items
    assert streams.fills_gpu(sh(128, 257))             # 256 items
    assert not streams.fills_gpu(sh(64, 1024))         # 32 x 4 = 128 items
    assert streams.fills_gpu(sh(64, 2048))             # 32 x 8 = 256 items
    assert not streams.fills_gpu(sh(64, 2048), nsm=300)
