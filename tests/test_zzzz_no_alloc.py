"""mc3_phase_shift_noalloc (fixed device scratch, no allocation) against
mc3_phase_shift, called through the C ABI.  Collected last (file name) so it
also runs after every other test in one process; it passes alone too."""
import ctypes

import numpy as np
import pytest

VP, I, F = ctypes.c_void_p, ctypes.c_int, ctypes.c_float
MC3_OK, MC3_ETOOBIG = 0, 7
MAX_CMP_X, MAX_CMP_Y = 8193, 16384


def _bind(lib):
    for name in ("mc3_phase_shift", "mc3_phase_shift_noalloc"):
        fn = getattr(lib, name)
        fn.argtypes = [VP, VP, I, I, F, F, I, VP]
        fn.restype = I
    return lib


def test_noalloc_rejects_sizes_above_its_scratch(mc3lib):
    L = _bind(mc3lib)
    dummy = ctypes.c_void_p(16)  # never dereferenced: the size check comes first
    assert L.mc3_phase_shift_noalloc(dummy, dummy, MAX_CMP_X + 1, 8, 1.0, 1.0, 0, None) == MC3_ETOOBIG
    assert L.mc3_phase_shift_noalloc(dummy, dummy, 65, MAX_CMP_Y + 1, 1.0, 1.0, 0, None) == MC3_ETOOBIG
    L.mc3_strerror.restype = ctypes.c_char_p
    L.mc3_strerror.argtypes = [I]
    assert b"scratch" in L.mc3_strerror(MC3_ETOOBIG)


@pytest.mark.gpu
def test_noalloc_matches_allocating_entry_point(mc3lib, torch_cuda):
    torch = torch_cuda
    L = _bind(mc3lib)
    rng = np.random.default_rng(77)
    # Two calls in a row on the same scratch: different sizes and shifts, the
    # second one accumulating; the second also reaches the maximum cmp_x.
    cases = [((384, 257), (3.37, -7.81), 0), ((96, MAX_CMP_X), (-12.5, 0.43), 1)]
    for (cy, cx), (sx, sy), acc in cases:
        X = (rng.standard_normal((cy, cx)) + 1j * rng.standard_normal((cy, cx))).astype(np.complex64)
        src = torch.from_numpy(X).cuda()
        init = torch.from_numpy(X[::-1].copy()).cuda()
        want = init.clone()
        got = init.clone()
        st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        assert L.mc3_phase_shift(VP(src.data_ptr()), VP(want.data_ptr()), cx, cy, sx, sy, acc, st) == MC3_OK
        assert L.mc3_phase_shift_noalloc(VP(src.data_ptr()), VP(got.data_ptr()), cx, cy, sx, sy, acc,
                                         st) == MC3_OK
        torch.cuda.synchronize()
        w, g = want.cpu().numpy(), got.cpu().numpy()
        # same tolerance as the phase-shift parity test (relative to the peak)
        assert np.abs(g - w).max() <= 1e-5 * np.abs(w).max()
