"""Sample lines of the reference's own output files (printed by Julia's println), kept as a
fixture for the output writers' number formatting. Run from the repository root:

    python tests/golden/make_output_lines.py /path/to/reference   (or set PTS_REFERENCE_DIR)

The fixture keeps every line of the short files (the iteration counts to tolerance per grid
size) and the first and last lines of the long ones; of the aspect-ratio sweep it also keeps
the rows with ny = 127 (nx 127, 255 and 511: nsub 1, 2 and 4, every fact). The oracle
reproduces the iteration totals of the first two grids in seconds; the batched sweep runs all
thirty rows in one launch.
"""
import glob
import json
import os
import sys


def main(ref):
    out = {}
    for path in sorted(glob.glob(os.path.join(ref, "output", "out_*.txt"))):
        lines = [ln.rstrip("\n") for ln in open(path) if ln.strip()]
        if lines:
            name = os.path.basename(path)
            keep = lines if len(lines) <= 12 else [lines[0], lines[-1]]
            if name == "out_Stokes2D_ve_aspect_ratio_param.txt":
                small = [ln for ln in lines
                         if ln.split()[:3] in (["127", "127", "1"], ["255", "127", "2"], ["511", "127", "4"])]
                keep = small + [ln for ln in keep if ln not in small]
            out[name] = keep
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_output_lines.json")
    json.dump(out, open(dst, "w"), indent=1)
    print(dst, sum(len(v) for v in out.values()), "lines")


def reference_dir():
    """The reference checkout: the first argument, else $PTS_REFERENCE_DIR."""
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PTS_REFERENCE_DIR")
    if not ref:
        sys.exit("usage: python tests/golden/make_output_lines.py /path/to/reference  (or set PTS_REFERENCE_DIR)")
    return ref


if __name__ == "__main__":
    main(reference_dir())
