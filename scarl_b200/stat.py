"""Stat_ScaRL's front end (SRC_F/Stat_ScaRL/main_Stat.f90:36-110) on one GPU.

The job list on standard input, as the reference reads it: the number of
files, calculateCorrL (0/1), deleteSampleInTheEnd (0/1), then per file its
path and the dataset name.  Each file gets its FP64 moments (and, with
calculateCorrL, spectra and correlation lengths written back into it) and a
STAT_<file> beside it.  With deleteSampleInTheEnd the sample's .h5 / .xmf
files (same stem) are removed afterwards, as the reference's
`rm <stem>*` does, restricted to those two extensions.
"""
import os
import sys

from . import api as S


def parse_jobs(text):
    tok = [t.strip().strip('"').strip("'") for t in text.split() if t.strip()]
    n, corr, delete = int(tok[0]), int(tok[1]), int(tok[2])
    files = [(tok[3 + 2 * i], tok[4 + 2 * i]) for i in range(n)]
    return corr == 1, delete == 1, files


def _delete_sample(res_path):
    folder = os.path.dirname(res_path) or "."
    stem = os.path.splitext(os.path.basename(res_path))[0]
    for f in os.listdir(folder):
        if f.startswith(stem) and f.endswith((".h5", ".xmf")) and not f.startswith("STAT_"):
            os.remove(os.path.join(folder, f))


def main(stream=None, ctx=None, out=None):
    stream = stream or sys.stdin
    out = out or sys.stdout
    corr, delete, files = parse_jobs(stream.read())
    own = ctx is None
    if own:
        ctx = S.Context(0)
    results = []
    try:
        for path, dset in files:
            avg, std, cl = S.stat_file(ctx, path, dset, corr)
            print(f"{path}: globalAvg = {avg:.15g} globalStdDev = {std:.15g}"
                  + ("" if cl is None else " corrL_out = " + " ".join(f"{v:.15g}" for v in cl)),
                  file=out)
            results.append((path, avg, std, cl))
            if delete:
                _delete_sample(path)
    finally:
        if own:
            ctx.close()
    return results


if __name__ == "__main__":
    main()
