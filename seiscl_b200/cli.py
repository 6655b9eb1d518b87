"""Command line of the engine: ``python -m seiscl_b200.cli [-p] <base> [din]``.

The counterpart of the reference's ``SeisCL_MPI [-p] <file> [<din file>]``
(src/SeisCL_MPI.c:33-161): it reads the job files ``<base>_csts.mat``,
``<base>_model.mat``, the observed data ``<base>_din.mat`` (or the file given
as second argument) and, for a gradient from given residuals,
``<base>_res.mat``; runs the forward modelling and, as the constants ask,
the residuals, misfit and adjoint gradient on the current CUDA device; and
writes ``<base>_dout.mat``, ``_gout.mat``, ``_rms.mat`` and ``_movie.mat``
beside them, with the datasets and layouts of src/writehdf5.c:190-316.  The
files are HDF5 (``seiscl_b200.h5lite``).

As SeisCL_MPI: the file list goes to standard output, an error is one line
on standard error and a nonzero exit status.  ``-p`` (print the generated
kernels) is accepted and has no effect: the kernels are compiled ahead of
time.  The job runs in the front end of ``seiscl_b200.seiscl``, the same
code the Python class runs in memory.
"""
from __future__ import annotations

import os
import sys


def main(argv=None) -> int:
    argv = list(sys.argv[1:] if argv is None else argv)
    opts = [a for a in argv if a.startswith("-") and len(a) > 1]
    pos = [a for a in argv if not (a.startswith("-") and len(a) > 1)]
    for o in opts:
        for ch in o[1:]:
            if ch == "h":
                sys.stdout.write("usage: python -m seiscl_b200.cli [-p] <base> [din]\n")
            elif ch != "p":
                sys.stderr.write("Unknown option character `\\x%x'.\n" % ord(ch))
                return 1
    if len(pos) > 2:
        sys.stderr.write("Too many default argument, expected 2\n")
        return 1
    filein = pos[0] if pos else "SeisCL"
    workdir, base = os.path.split(filein)
    workdir = workdir or "."
    try:
        from .seiscl import SeisCL, SeisCLError
    except Exception as exc:   # the engine library could not be loaded
        sys.stderr.write("Error: %s\n" % exc)
        return 1
    try:
        s = SeisCL(file=base, workdir=workdir, files=True)
        if len(pos) > 1:
            s.file_din = os.path.abspath(pos[1])
        sys.stdout.write("\nInput files for SeisCL: \n")
        for what, name in (("model", s.file_model), ("constants", s.file_csts), ("output data", s.file_dout),
                           ("output gradient", s.file_gout), ("output rms", s.file_rms),
                           ("output movie", s.file_movout), ("input data", s.file_din)):
            sys.stdout.write("    %s: %s \n" % (what, s._path(name)))
        s.read_csts()
        log = s.execute()
        sys.stdout.write(log)
        s.close()
    except SeisCLError as exc:
        msg = str(exc).strip() or "Error"
        sys.stderr.write(msg + "\n")
        return 1
    return 0


if __name__ == "__main__":
    sys.exit(main())
