"""Golden initial conditions from the reference's own generator.

    python tests/golden/make_ic_golden.py run --out DIR        (on a machine with a GPU)
    python tests/golden/make_ic_golden.py package --src DIR    (anywhere)

`run` executes ``oracle/_ref/<cfg>/refdrv ic`` for the configurations below:
the reference's initializeJet (initialize.cu:615-641: generateNoise with its
rand() stream, the tanh jet and scalar profiles, pert_amp 0.05), forward
transforms and deAlias, exactly as main.cu:139-156, built from the unmodified
sources by oracle/build_ref.sh.  `package` turns the dumps into
tests/golden/ic_<cfg>.npz (the five spectral fields and the parameters).
"""
from __future__ import annotations

import argparse
import subprocess
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
# name: (N, H, theta, theta_c, pert_amp) as generated into dnsparams.h by oracle/build_ref.sh
CONFIGS = {"i16": (16, 1.0, 0.05, 0.05, 0.05), "i32": (32, 1.0, 0.05, 0.05, 0.05)}


def run(out: Path) -> None:
    for name in CONFIGS:
        d = out / name
        d.mkdir(parents=True, exist_ok=True)
        exe = ROOT / "oracle" / "_ref" / name / "refdrv"
        subprocess.run([str(exe), "ic", str(d)], check=True, stdout=subprocess.DEVNULL)


def package(src: Path) -> None:
    for name, (n, h, theta, theta_c, pert) in CONFIGS.items():
        raw = np.fromfile(src / name / "ic.bin", dtype=np.complex128)
        fields = raw.reshape(5, n, n, n // 2 + 1)
        np.savez_compressed(HERE / f"ic_{name}.npz", fields=fields, n=n, h=h, theta=theta, theta_c=theta_c,
                            pert_amp=pert)
        print(f"wrote ic_{name}.npz")


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("step", choices=("run", "package"))
    ap.add_argument("--out", help="directory for the reference's dumps (step run)")
    ap.add_argument("--src", help="directory holding those dumps (step package)")
    a = ap.parse_args()
    if (a.out if a.step == "run" else a.src) is None:
        ap.error("run needs --out, package needs --src")
    if a.step == "run":
        run(Path(a.out))
    else:
        package(Path(a.src))
    return 0


if __name__ == "__main__":
    sys.exit(main())
