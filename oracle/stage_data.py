"""Copy the reference's radiation data files into <repo>/data (git-ignored).

A build step: __graft_entry__.build() runs it with the reference checkout's
run/data directory where that checkout exists; the copied files then travel
with the working tree.  The source directory is the first argument, else the
MGCM_RT_REFERENCE_DATA environment variable; with neither, nothing is staged.

    python oracle/stage_data.py SOURCE_DIR
"""
import os
import pathlib
import shutil
import sys

FILES = ("CO2H2O_V_12_95_INTEL", "CO2H2O_IR_12_95_INTEL",
         "waterCoated_vis_JD_12bands.dat", "waterCoated_ir_JD_12bands.dat",
         "Dust_vis_wolff2010_JD_12bands.dat", "Dust_ir_wolff2010_JD_12bands.dat")
DST = pathlib.Path(__file__).resolve().parents[1] / "data"


def stage(src: pathlib.Path, dst: pathlib.Path = DST) -> bool:
    if not all((src / f).is_file() for f in FILES):
        return False
    dst.mkdir(parents=True, exist_ok=True)
    for f in FILES:
        if not (dst / f).is_file() or (dst / f).stat().st_size != (src / f).stat().st_size:
            shutil.copyfile(src / f, dst / f)
    return True


if __name__ == "__main__":
    src = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("MGCM_RT_REFERENCE_DATA")
    ok = bool(src) and stage(pathlib.Path(src))
    print("staged" if ok else "source data not found; nothing staged")
