"""``python -m canard_b200.dcanard -d DIR1 DIR2 [-t TOL]``: the reference's
restart comparer (contrib/dcanard.f90, contrib/dcanard). It reads the block
sizes from ``input.canard`` in the current directory (nml_driver,
nml_domdcomp), compares each block's restart file ``misc/restartzNNN.da`` of
the two run directories point by point and variable by variable with the
relative tolerance TOL (default 1e-15), writes the differences to
``output/restartN.dat`` (N = block, one line per value beyond the tolerance,
in the reference's format) and prints ``Compared <points> elements for 5
variables in block N``. Exit status 0 when every block's files read."""
import argparse
import os
import sys

from . import api, namelist


def compare(dir1: str, dir2: str, tol: float = 1.0e-15, input_path: str = "input.canard",
            report_dir: str = "output", out=sys.stdout) -> int:
    """Compares every block; returns the number of values beyond the tolerance."""
    nml = namelist.read_file(input_path)
    dd = nml["nml_domdcomp"]
    nb = int(nml["nml_driver"]["mbk"]) + 1
    os.makedirs(report_dir, exist_ok=True)
    print(" Command line arguments:", file=out)
    print(" directory 1: ", dir1, file=out)
    print(" directory 2: ", dir2, file=out)
    print(" tolerance  : ", tol, file=out)
    total = 0
    for mb in range(nb):
        npts = int((dd["lximb"][0][mb] + 1) * (dd["letmb"][0][mb] + 1) * (dd["lzemb"][0][mb] + 1))
        total += api.compare_restart(os.path.join(dir1, api.restart_name(mb)), os.path.join(dir2, api.restart_name(mb)),
                                     npts, tol, report=os.path.join(report_dir, "restart%d.dat" % mb))
        print("Compared %8d elements for %8d variables in block %8d" % (npts, 5, mb), file=out)
    return total


def main(argv=None):
    p = argparse.ArgumentParser(prog="python -m canard_b200.dcanard",
                                description="compare the restart files of two run directories")
    p.add_argument("-d", "--directories", nargs=2, required=True, metavar=("DIR1", "DIR2"))
    p.add_argument("-t", "--tolerance", type=float, default=1.0e-15)
    p.add_argument("--input", default="input.canard")
    a = p.parse_args(argv)
    compare(a.directories[0], a.directories[1], a.tolerance, a.input)
    return 0


if __name__ == "__main__":
    sys.exit(main())
