"""Command-line entry points equivalent to the reference's ed.x / xas.x / rixs.x / opavg.x.

The reference installs them as console scripts (setup.py:101-108 -> edrixs/scripts.py:1-46)
that take MPI.COMM_WORLD and call the f2py solvers in the working directory.  These run the
B200 solvers on the files of the working directory; under a multi-process launcher only
rank 0 works (the others return), as the drop-in solvers document.

    python -m edrixs_b200.scripts ed|xas|rixs|opavg
"""
import os
import sys

from . import fedrixs


def _rank():
    for var in ("RANK", "OMPI_COMM_WORLD_RANK", "PMI_RANK"):
        if var in os.environ:
            return int(os.environ[var])
    return 0


def ed():
    fedrixs.ed_fsolver(0, _rank(), 1)


def xas():
    fedrixs.xas_fsolver(0, _rank(), 1)


def rixs():
    fedrixs.rixs_fsolver(0, _rank(), 1)


def opavg():
    fedrixs.opavg_fsolver(0, _rank(), 1)


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    cmds = {"ed": ed, "xas": xas, "rixs": rixs, "opavg": opavg}
    if len(argv) != 1 or argv[0] not in cmds:
        print("usage: python -m edrixs_b200.scripts ed|xas|rixs|opavg", file=sys.stderr)
        return 2
    cmds[argv[0]]()
    return 0


if __name__ == "__main__":
    sys.exit(main())
