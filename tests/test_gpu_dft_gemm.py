"""Split-precision BF16 DFT GEMMs on the tensor cores (tcgen05.mma, FP32
accumulation in tensor memory) against FP64 references.

* Row transforms (mc3_rfft_rows, method 1) of 408- and 410-point rows (the
  patch sizes of the benchmark and of 5760x4092 movies) and other even
  lengths against numpy's FP64 rfft: the error is stated per case and held
  to 3e-5 of the spectrum maximum (the FP32 FFT: 2e-6).
* The patch path with the GEMM row transforms (mc3_params.dft_gemm = 1)
  against the FP64 oracle: patch and global shifts within 0.05 px, sums of
  the oracle corrected with the same shifts within 1e-4 relative RMS, and
  the shifts' distance from the FP32 path's stated.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def api(mc3lib, torch_cuda):
    from motioncor3_b200 import api as A
    return A


@pytest.mark.parametrize("nx,rows,pitch", [(408, 1000, 410), (410, 300, 412), (64, 129, 64),
                                           (256, 513, 260), (414, 128, 414)])
def test_rfft_rows_split_bf16_gemm(api, torch_cuda, nx, rows, pitch):
    torch = torch_cuda
    rng = np.random.default_rng(nx + rows)
    x = rng.poisson(3.0, (rows, pitch)).astype(np.float32) * rng.uniform(0.9, 1.1, (rows, pitch)).astype(np.float32)
    ref = np.fft.rfft(x[:, :nx].astype(np.float64), axis=1)
    src = torch.from_numpy(x).cuda()
    out = {}
    for method in (0, 1):
        dst = torch.zeros((rows, nx // 2 + 1), dtype=torch.complex64, device="cuda")
        api.rfft_rows(src, dst, nx, method)
        torch.cuda.synchronize()
        got = dst.cpu().numpy().astype(np.complex128)
        err = np.abs(got - ref)
        out[method] = (err.max() / np.abs(ref).max(),
                       np.sqrt(np.mean(err ** 2) / np.mean(np.abs(ref) ** 2)))
    print(f"{nx}-point rows x {rows}: FP32 FFT max {out[0][0]:.1e} rms {out[0][1]:.1e}; "
          f"split-BF16 GEMM max {out[1][0]:.1e} rms {out[1][1]:.1e}")
    assert out[0][0] < 2e-6
    assert out[1][0] < 3e-5 and out[1][1] < 1e-5


def test_patch_path_with_dft_gemm_against_oracle(api, oracle, torch_cuda):
    from motioncor3_b200 import synthetic as S
    m = S.make_movie(2048, 2048, 10, dose=1.0, seed=71, gain=True, local=True)
    frames, gain = np.asarray(m.frames), np.asarray(m.gain)
    common = dict(patch=(5, 5), iter=10, tol=0.1, bft=(500, 150), fm_dose=1.2, pix_size=1.0, kv=300)
    res = {}
    for form in (0, 1):
        with api.MotionCor3(api.Params(dft_gemm=form, **common)) as mc:
            mc.set_gain(gain)
            info = mc.plan(2048, 2048, 10)
            res[form] = mc.process(frames)
    assert info["patch_size"] == (408, 408)
    orc = oracle.process_movie(frames, gain=gain, **common)
    r = res[1]
    dg = float(np.abs(r.global_shifts - orc["global_shifts"]).max())
    dp = float(np.abs(r.patch_shifts - orc["patch_shifts"]).max())
    dplain = float(np.abs(r.patch_shifts - res[0].patch_shifts).max())
    print(f"split-BF16 patch transforms: patch shifts max |d| {dp:.4f} px against the FP64 oracle, "
          f"{dplain:.4f} px against the FP32 path; global {dg:.4f} px")
    assert dg <= 0.05 and dp <= 0.05
    assert np.array_equal(r.patch_centers, orc["patch_centers"])
    force = dict(global_shifts=r.global_shifts, patch_shifts=r.patch_shifts,
                 patch_centers=r.patch_centers, patch_bad=r.patch_bad)
    same = oracle.process_movie(frames, gain=gain, force=force, **common)
    for s in range(r.n_sums):
        a = r.sums[s].astype(np.float64)
        b = same["sums"][s].astype(np.float64)
        e = float(np.sqrt(np.mean((a - b) ** 2) / np.mean(b ** 2)))
        print(f"  sum {s}: rel RMS {e:.2e} against the oracle with the same shifts")
        assert e <= 1e-4, (s, e)
