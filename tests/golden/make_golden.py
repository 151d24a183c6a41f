"""Extract the reference's golden vectors into tests/golden/golden.json.

Run once where the reference tree exists, giving its path as the argument
or in $GEMS_REF; the resulting JSON is committed so the tests never read the
reference at run time.  It collects the regression outputs that pin the
force/neighbour path (examples/*/ref/Energy.*.dat, the test rule of
examples/test.sh) and the input coordinates those decks read.

    python tests/golden/make_golden.py [/path/to/GEMS]
"""
import json
import os
import sys

REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("GEMS_REF")
if not REF:
    sys.exit("usage: make_golden.py /path/to/GEMS   (or set GEMS_REF)")
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden.json")


def rows(path):
    with open(os.path.join(REF, path)) as f:
        return [[float(t) for t in line.split()] for line in f if line.strip()]


def xyz_frames(path):
    """All frames of an xyz file as lists of [x, y, z]."""
    frames = []
    with open(os.path.join(REF, path)) as f:
        lines = [ln.rstrip("\n") for ln in f]
    k = 0
    while k < len(lines):
        if not lines[k].strip():
            k += 1
            continue
        n = int(lines[k].split()[0])
        body = lines[k + 2: k + 2 + n]
        frames.append([[float(t) for t in ln.split()[1:4]] for ln in body])
        k += 2 + n
    return frames


def main():
    g = {
        "source": "alexispaz/GEMS examples/*/ref (regression outputs, printed E15.7)",
        "rule": "examples/test.sh: abs(sum((ref1-new1)^2)/sum(ref1)) < 1e-6 on column 1",
        "xyz_frames": xyz_frames("examples/XYZ/Pos.md.xyz"),
        "xyz_energy": rows("examples/XYZ/ref/Energy.readxyz.dat"),
        "lj_energy": rows("examples/LJ/ref/Energy.lj.dat"),
        "slj_energy": rows("examples/LJ/ref/Energy.slj.dat"),
        "wca_energy": rows("examples/LJ/ref/Energy.wca.dat"),
        "sm1_energy": rows("examples/LJ/ref/Energy.sm1.dat"),
        "feels_energy": rows("examples/LJ/ref/Energy.feels.dat"),
        "smatb_md_coords": xyz_frames("examples/SMA-TB/coords.xyz")[0],
        "smatb_md_energy": rows("examples/SMA-TB/ref/Energy.md.dat"),
        "smatb_bulk_energy": rows("examples/SMA-TB/ref/Energy.bulk.dat"),
        "nve_energy": rows("examples/NVE/ref/Energy.v_verlet.dat"),
        "nve_pc5_energy": rows("examples/NVE/ref/Energy.pred_corr_5.dat"),
        "nvt_energy": rows("examples/NVT/ref/Energy.ermak.dat"),
        "repex_energy": [rows("examples/RepExchange/ref/Energy.lj.mpi%d.dat" % k) for k in range(4)],
        "neb_gold_cube": xyz_frames("examples/configs/ref/gold_cube.xyz")[0],
        "neb_energy": rows("examples/NEB/ref/Energy.neb.dat.NebF"),
        "npt_lgf_energy": rows("examples/NPT/ref/Energy.lgf.dat"),
        "npt_lgf_press": rows("examples/NPT/ref/Press.lgf.dat"),
        "npt_lgf_virial": rows("examples/NPT/ref/Viri.lgf.dat"),
        "npt_flex_energy": rows("examples/NPT/ref/Energy.lgf_flex.dat"),
        "npt_flex_press": rows("examples/NPT/ref/Press.lgf_flex.dat"),
        "npt_flex_virial": rows("examples/NPT/ref/Viri.lgf_flex.dat"),
        "npt_x_energy": rows("examples/NPT/ref/Energy.lgf_x.dat"),
        "npt_x_press": rows("examples/NPT/ref/Press.lgf_x.dat"),
        "npt_x_box": rows("examples/NPT/ref/Caja.lgf_x.dat"),
    }
    with open(OUT, "w") as f:
        json.dump(g, f)
    print("wrote", OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    main()
