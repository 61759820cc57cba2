"""Golden files of the reference's own writers (iofuncs.cu), for the byte-exact
tests of the library's reference-format I/O.

    python tests/golden/make_io_golden.py

Runs ``oracle/_ref/g12/refdrv io`` (built from the unmodified reference
sources by oracle/build_ref.sh; its io mode calls write3Dfields_mgpu,
writexyfields, writexzfields, writeyzfields, writeStats and writeYprofs on a
synthetic 12^3 field, host code only) in a temporary directory and copies its
output into tests/golden/io_g12/.
"""
from __future__ import annotations

import shutil
import subprocess
import sys
import tempfile
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
EXE = ROOT / "oracle" / "_ref" / "g12" / "refdrv"
OUT = HERE / "io_g12"
FILES = ["u.3", "vis/u_xy.3", "vis/u_xz.3", "vis/u_yz.3", "stats/KE", "Yprofs/u_mean.3", "input.bin", "prof.bin"]


def main() -> int:
    if not EXE.exists():
        subprocess.run(["bash", str(ROOT / "oracle" / "build_ref.sh"), "g12"], check=True)
    with tempfile.TemporaryDirectory() as tmp:
        subprocess.run([str(EXE), "io"], cwd=tmp, check=True, stdout=subprocess.DEVNULL)
        if OUT.exists():
            shutil.rmtree(OUT)
        for f in FILES:
            dst = OUT / f
            dst.parent.mkdir(parents=True, exist_ok=True)
            shutil.copyfile(Path(tmp) / "refdrv" / f, dst)
    print(f"wrote {len(FILES)} files to {OUT}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
