"""Times the reference program (built by this directory's Makefile) and the
mc3-b200 command line on the same synthetic movie on one GPU, and records
both programs' printed "Computation time" (gain -> bad pixels -> align ->
sums, CProcessThread.cpp:103-104) plus wall time.  Checker / baseline tool,
run on a machine with a GPU:

  python oracle/ref_full/time_reference.py --config cfg2 --out ref_cfg2.json
"""
import argparse
import json
import os
import re
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

CONFIGS = {
    "cfg1": dict(shape=(40, 1024, 1024), dose=1.0, gain=False, local=False,
                 tags="-Patch 0 0 -Iter 7 -Tol 0.5 -Bft 150 -PixSize 1.0"),
    "cfg2": dict(shape=(60, 4096, 4096), dose=0.8, gain=True, local=True,
                 tags="-Patch 5 5 -Iter 10 -Bft 500 150 -FmDose 1.161 -PixSize 0.83 -kV 300"),
}


def run(binary, workdir, movie_path, gain_path, tags):
    args = [binary, "-InMrc", movie_path, "-OutMrc", os.path.join(workdir, "sum.mrc"), "-LogDir",
            workdir + "/", "-Gpu", "0", "-Cs", "0"] + tags.split()
    if gain_path:
        args += ["-Gain", gain_path]
    env = dict(os.environ)
    env["LD_LIBRARY_PATH"] = "/usr/local/cuda/lib64:" + env.get("LD_LIBRARY_PATH", "")
    t0 = time.time()
    p = subprocess.run(args, capture_output=True, text=True, env=env, timeout=1800, cwd=workdir)
    wall = time.time() - t0
    out = p.stdout + p.stderr
    m = re.search(r"Computation time:\s*([0-9.]+)", out)
    return dict(rc=p.returncode, computation_s=float(m.group(1)) if m else None, wall_s=wall,
                tail=out[-1500:])


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", default="cfg1", choices=list(CONFIGS))
    ap.add_argument("--work", default="/tmp/mc3_ref_timing")
    ap.add_argument("--out", default=None)
    ap.add_argument("--repeat", type=int, default=2)
    a = ap.parse_args()
    import numpy as np
    import torch
    from motioncor3_b200 import mrcio, synthetic as S
    c = CONFIGS[a.config]
    nz, ny, nx = c["shape"]
    os.makedirs(a.work, exist_ok=True)
    m = S.make_movie(nx, ny, nz, dose=c["dose"], seed=5, gain=c["gain"], local=c["local"],
                     backend="torch")
    mp = os.path.join(a.work, "movie.mrc")
    mrcio.write(mp, m.frames.cpu().numpy())
    gp = None
    if m.gain is not None:
        gp = os.path.join(a.work, "gain.mrc")
        mrcio.write(gp, m.gain.cpu().numpy())
    del m
    torch.cuda.empty_cache()
    res = {"config": a.config, "frames": nz, "size": [nx, ny], "tags": c["tags"]}
    for name, binary in (("reference", os.path.join(ROOT, "oracle", "_ref", "MotionCor3")),
                         ("mc3_b200_cli", os.path.join(ROOT, "motioncor3_b200", "MotionCor3"))):
        runs = []
        for r in range(a.repeat):
            wd = os.path.join(a.work, f"{name}_{r}")
            os.makedirs(wd, exist_ok=True)
            runs.append(run(binary, wd, mp, gp, c["tags"]))
        res[name] = runs
        best = [x["computation_s"] for x in runs if x["computation_s"]]
        if best:
            res[name + "_frames_per_s"] = nz / min(best)
    txt = json.dumps(res, indent=1)
    print(txt)
    if a.out:
        open(a.out, "w").write(txt)


if __name__ == "__main__":
    main()
