"""Given patch centres (mc3_set_patch_centers, command line -PatchCenters):
the conversion from full-frame centres to patch starts in the alignment
image, on the CPU (mc3_patch_starts_from_centers, the engine's own code)."""
import numpy as np
import pytest

# (alignment image, xcf bin, patch size) of the 4096^2 and 5760x4092 movies
GEOMETRIES = [((2048, 2048), (2.0, 2.0), (408, 408)),
              ((2882, 2048), (2880.0 / 1441.0, 4092.0 / 2048.0), (410, 408)),
              ((1024, 1024), (1.0, 1.0), (204, 204))]


@pytest.mark.parametrize("xcf,bins,pat", GEOMETRIES)
def test_reported_centres_give_back_their_starts(mc3lib, xcf, bins, pat):
    """The centres the engine reports ((start + size/2) * bin, as the logs
    print them to 0.01 px) lead back to the same patch starts, so a run at
    another run's logged centres cuts the same patches."""
    from motioncor3_b200 import api
    rng = np.random.default_rng(xcf[0])
    starts = np.stack([rng.integers(0, xcf[0] - pat[0] + 1, 200),
                       rng.integers(0, xcf[1] - pat[1] + 1, 200)], axis=1)
    centres = ((starts + np.array(pat) // 2) * np.array(bins, np.float32)).astype(np.float32)
    logged = np.round(centres.astype(np.float64), 2)  # "%.2f" in the patch log
    got = api.patch_starts_from_centers(logged, bins, xcf, pat)
    assert np.array_equal(got, starts)


def test_centres_outside_keep_the_patch_inside(mc3lib):
    from motioncor3_b200 import api
    xcf, bins, pat = GEOMETRIES[0]
    c = np.array([[-500.0, 10.0], [5000.0, 8000.0], [0.0, 4095.0]], np.float32)
    got = api.patch_starts_from_centers(c, bins, xcf, pat)
    assert got.tolist() == [[0, 0], [xcf[0] - pat[0], xcf[1] - pat[1]], [0, xcf[1] - pat[1]]]


def test_bad_arguments_are_refused(mc3lib):
    from motioncor3_b200 import api
    c = np.array([[100.0, 100.0]], np.float32)
    for args in [((0.0, 2.0), (2048, 2048), (408, 408)), ((2.0, 2.0), (300, 2048), (408, 408))]:
        with pytest.raises(api.MC3Error):
            api.patch_starts_from_centers(c, *args)
    with pytest.raises(api.MC3Error):
        api.patch_starts_from_centers(np.array([[np.nan, 1.0]], np.float32), (2.0, 2.0),
                                      (2048, 2048), (408, 408))
