"""The movie queue (mc3_submit / mc3_wait): movies of uneven size and frame
count, submitted back to back from pinned host memory, are processed in
order on the context's worker thread, each one's copy overlapping the
previous one's kernels; every result is identical, bit for bit, to
processing the same movie alone with mc3_process_movie."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SHAPES = [(256, 256, 10), (384, 320, 14), (512, 512, 8), (256, 256, 20), (320, 384, 9)]


def _movies():
    from motioncor3_b200 import synthetic as S
    return [S.make_movie(nx, ny, nz, dose=3.0, seed=90 + i, local=True)
            for i, (nx, ny, nz) in enumerate(SHAPES)]


@pytest.mark.parametrize("patch", [(0, 0), (3, 3)])
def test_queue_matches_single_movies(mc3lib, torch_cuda, patch):
    torch = torch_cuda
    from motioncor3_b200 import api
    movies = _movies()
    p = api.Params(patch=patch, iter=6, tol=0.2, bft=(300, 150), fm_dose=1.0, pix_size=1.0)
    with api.MotionCor3(p) as mc:
        alone = [mc.process(m.frames) for m in movies]
    pinned = [torch.from_numpy(m.frames).pin_memory() for m in movies]
    with api.MotionCor3(p) as mc:
        tickets = [mc.submit(f.numpy()) for f in pinned]
        done = [mc.wait(t) for t in tickets]
    lat = [d[1] for d in done]
    print(f"patch {patch}: latencies (ms, submit to done) {[round(x, 2) for x in lat]}")
    assert all(b > a for a, b in zip(lat, lat[1:]))  # processed in submission order
    for a, (b, _) in zip(alone, done):
        assert np.array_equal(a.global_shifts, b.global_shifts)
        if a.n_patches:
            assert np.array_equal(a.patch_shifts, b.patch_shifts)
        for s in range(a.n_sums):
            assert np.array_equal(a.sums[s], b.sums[s])


def test_queue_reports_a_failed_movie_and_continues(mc3lib, torch_cuda):
    from motioncor3_b200 import api
    movies = _movies()[:3]
    p = api.Params(iter=5, tol=0.2, bft=(300, 150), pix_size=1.0)
    with api.MotionCor3(p) as mc:
        mc.set_gain(np.ones((256, 256), np.float32))  # fits the first movie only
        t = [mc.submit(m.frames) for m in movies]
        first, _ = mc.wait(t[0])
        with pytest.raises(api.MC3Error):
            mc.wait(t[1])            # 384 x 320 against a 256 x 256 gain
        with pytest.raises(api.MC3Error):
            mc.wait(t[2])
        mc.set_gain(None)
        again = mc.process(movies[0].frames)
    assert np.array_equal(first.global_shifts, again.global_shifts)


def test_autotune_writes_and_loads_its_choice(mc3lib, torch_cuda, tmp_path):
    """mc3_autotune times all 8 variants on a synthetic movie of the size,
    keeps the fastest and writes every time to the JSON file; a new context
    loads the file and processes movies of that size with the choice."""
    import json
    from motioncor3_b200 import api, synthetic as S
    path = str(tmp_path / "tuning.json")
    p = api.Params(patch=(3, 3), iter=5, tol=0.2, bft=(500, 150), pix_size=1.0)
    with api.MotionCor3(p) as mc:
        best = mc.autotune(512, 512, 10, path)
        mc.autotune(256, 256, 12, path)   # a second size joins the file
    doc = json.load(open(path))
    e = [x for x in doc["entries"] if x["nx"] == 512][0]
    assert len(doc["entries"]) == 2 and len(e["candidates"]) == 8
    assert e["ms"] == pytest.approx(best, rel=1e-3)
    assert e["ms"] == pytest.approx(min(c["ms"] for c in e["candidates"]), rel=1e-3)
    m = S.make_movie(512, 512, 10, dose=3.0, seed=97, local=True)
    with api.MotionCor3(p) as mc:
        plain = mc.process(m.frames)
    with api.MotionCor3(p) as mc:
        mc.load_tuning(path)
        tuned = mc.process(m.frames)
    assert np.abs(tuned.global_shifts - plain.global_shifts).max() <= 0.05
    for s in range(plain.n_sums):
        a, b = tuned.sums[s].astype(np.float64), plain.sums[s].astype(np.float64)
        assert np.sqrt(np.mean((a - b) ** 2) / np.mean(b ** 2)) <= 1e-3
