"""mc3_prefetch_movie: movies whose raw frames were copied ahead on the copy
stream give the same results as plain mc3_process_movie calls, and the
order rule is enforced."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_prefetched_movies_match_plain_calls(torch_cuda):
    torch = torch_cuda
    from motioncor3_b200 import api, synthetic as S
    movies = [S.make_movie(384, 320, 10, dose=3.0, seed=70 + i, gain=False, local=False).frames
              for i in range(3)]
    pinned = [torch.from_numpy(m).pin_memory().numpy() for m in movies]
    p = api.Params(patch=(0, 0), iter=6, tol=0.2, bft=(300, 100), fm_dose=1.0, pix_size=1.0)
    with api.MotionCor3(p) as mc:
        plain = [mc.process(m) for m in pinned]
        mc.prefetch(pinned[0])
        mc.prefetch(pinned[1])
        with pytest.raises(api.MC3Error):
            mc.prefetch(pinned[2])          # at most two outstanding
        with pytest.raises(api.MC3Error):
            mc.process(pinned[2])           # not the oldest prefetched movie
        got = [mc.process(pinned[0])]
        mc.prefetch(pinned[2])
        got.append(mc.process(pinned[1]))
        got.append(mc.process(pinned[2]))
    for a, b in zip(plain, got):
        assert np.array_equal(a.global_shifts, b.global_shifts)
        assert np.array_equal(a.sums, b.sums)
