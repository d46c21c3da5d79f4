"""The three 4096-point column passes (MC3_FFT_COL_WIDE = 0: two columns per
CTA, 1: four columns per CTA, 2: persistent CTAs that prefetch the next
four columns with cp.async while transforming the current ones) and the two
4096-real row R2C passes (MC3_FFT_ROW_PIPE = 0: one load phase per CTA, 1:
persistent CTAs whose next rows arrive by bulk copies on an mbarrier) run
the same radix-16 arithmetic in the same order, so their results are
identical bit for bit: the forward and inverse transforms of 4096^2 frames
(checked against FP64 numpy as well) and a whole 4096^2 movie with 5x5
patches (shifts and sums).  Each variant runs in its own process, since the
default is read from the environment once per process."""
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# (MC3_FFT_COL_WIDE, MC3_FFT_ROW_PIPE)
VARIANTS = [(1, 0), (0, 0), (2, 0), (2, 1)]

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = r"""
import sys
import numpy as np
import torch
sys.path.insert(0, sys.argv[1])
from motioncor3_b200 import api
from motioncor3_b200 import synthetic as S
out = sys.argv[2]
rng = np.random.default_rng(4096)
nz, n = 3, 4096
img = rng.standard_normal((nz, n, n)).astype(np.float32)
cx = n // 2 + 1
buf = torch.zeros((nz, n, 2 * cx), dtype=torch.float32, device="cuda")
buf[:, :, :n] = torch.from_numpy(img).cuda()
api.fft_forward(buf, n, n, normalise=True)
spec = buf.cpu().numpy()
half = (rng.standard_normal((nz, n, cx)) + 1j * rng.standard_normal((nz, n, cx))).astype(np.complex64)
hb = torch.view_as_real(torch.from_numpy(half).cuda()).reshape(nz, n, 2 * cx).contiguous()
api.fft_inverse(hb, n, n)
inv = hb[:, :, :n].cpu().numpy()
mv = S.make_movie(n, n, 8, dose=2.0, seed=77, gain=True, local=True)
p = api.Params(patch=(5, 5), iter=10, tol=0.1, bft=(500, 150), fm_dose=1.161, pix_size=0.83, kv=300)
with api.MotionCor3(p) as mc:
    mc.set_gain(mv.gain)
    r = mc.process(mv.frames)
np.savez(out, spec=spec, inv=inv, img0=img[0], gsh=r.global_shifts, psh=r.patch_shifts,
         sums=r.sums)
"""


@pytest.fixture(scope="module")
def variants(mc3lib, tmp_path_factory):
    d = tmp_path_factory.mktemp("colvar")
    script = d / "run.py"
    script.write_text(SCRIPT)
    res = {}
    for w in VARIANTS:
        col, row = w
        env = dict(os.environ, MC3_FFT_COL_WIDE=str(col), MC3_FFT_ROW_PIPE=str(row),
                   MC3_FFT_R16="1")
        out = d / f"v{col}{row}.npz"
        p = subprocess.run([sys.executable, str(script), ROOT, str(out)], env=env,
                           capture_output=True, text=True, timeout=900)
        assert p.returncode == 0, p.stderr[-2000:]
        res[w] = dict(np.load(out))
    return res


def test_forward_transform_against_fp64(variants):
    v = variants[(2, 1)]
    n, cx = 4096, 2049
    spec = v["spec"][0].view(np.complex64)[:, :cx]
    ref = np.fft.rfft2(v["img0"].astype(np.float64)) / (n * n)
    err = np.abs(spec - ref).max() / np.abs(ref).max()
    print(f"persistent column and row passes, 4096^2 forward: {err:.2e} of the spectrum maximum")
    assert err < 2e-6


@pytest.mark.parametrize("key", ["spec", "inv", "gsh", "psh", "sums"])
def test_column_variants_identical(variants, key):
    a = variants[VARIANTS[0]][key]
    for w in VARIANTS[1:]:
        assert np.array_equal(variants[w][key], a), (w, key)
