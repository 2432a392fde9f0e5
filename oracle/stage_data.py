"""Copy the reference's radiation data files into <repo>/data (git-ignored).

A build step, run by __graft_entry__.build() in the container that holds the
reference checkout; the copied files then travel with the working tree.  The
source defaults to the reference checkout's run/data directory.

    python oracle/stage_data.py [SOURCE_DIR]
"""
import pathlib
import shutil
import sys

FILES = ("CO2H2O_V_12_95_INTEL", "CO2H2O_IR_12_95_INTEL",
         "waterCoated_vis_JD_12bands.dat", "waterCoated_ir_JD_12bands.dat",
         "Dust_vis_wolff2010_JD_12bands.dat", "Dust_ir_wolff2010_JD_12bands.dat")
DEFAULT_SRC = pathlib.Path("/root/reference/run/data")
DST = pathlib.Path(__file__).resolve().parents[1] / "data"


def stage(src: pathlib.Path = DEFAULT_SRC, dst: pathlib.Path = DST) -> bool:
    if not all((src / f).is_file() for f in FILES):
        return False
    dst.mkdir(parents=True, exist_ok=True)
    for f in FILES:
        if not (dst / f).is_file() or (dst / f).stat().st_size != (src / f).stat().st_size:
            shutil.copyfile(src / f, dst / f)
    return True


if __name__ == "__main__":
    ok = stage(pathlib.Path(sys.argv[1]) if len(sys.argv) > 1 else DEFAULT_SRC)
    print("staged" if ok else "source data not found; nothing staged")
