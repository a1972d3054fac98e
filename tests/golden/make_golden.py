"""Regenerate tests/golden/*.json from the reference's own regression fixtures.

The reference (PTsolvers/PseudoTransientStokes.jl) pins its solvers with six BSON
files under test/reftest-files/ (written by ReferenceTests.jl, compared with
``isapprox``; test/test_2D.jl:35-39, test/test_3D_{1,2,3}.jl). Each holds
``{P: Float64 array, X: Float64 vector}``: the pressure ``Pt`` and the cell-centre
coordinates ``xc`` sampled at ``Int.(ceil.(LinRange(1, n, 12)))`` per dimension.

This script decodes those files (BSON: int32 document length, typed elements;
ReferenceTests stores an array as ``{tag, type, size, data}`` with little-endian
column-major bytes) and writes each as JSON with exact hex floats, plus the run
that produced it. It reads the reference checkout, so it runs only where that
checkout exists; the JSON files it writes are committed.

    python tests/golden/make_golden.py /path/to/reference   (or set PTS_REFERENCE_DIR)
"""
import hashlib
import json
import os
import struct
import sys

HERE = os.path.dirname(os.path.abspath(__file__))

# fixture -> (reference script, oracle variant, grid, run description)
RUNS = {
    "test_Stokes_2D_v.bson": ("scripts/Stokes2D.jl", "2d_v", [63, 63], "converged to 1e-8, nout=500"),
    "test_Stokes_2D_ve.bson": ("scripts/Stokes2D_ve.jl", "2d_ve", [63, 63], "5 physical steps, each to 1e-8"),
    "test_Stokes_2D_ve_perf.bson": ("scripts/Stokes2D_ve_perf.jl", "2d_ve_perf", [63, 63], "nt=1, 101 PT iterations"),
    "test_Stokes3D_ve_multixpu.bson": ("scripts/stokes_3D/Stokes3D_ve_multixpu.jl", "3d_ve", [31, 31, 31],
                                       "1 rank, 5 physical steps, each to 1e-8"),
    "test_Stokes3D_ve_multixpu_perf.bson": ("scripts/stokes_3D/Stokes3D_ve_multixpu_perf.jl", "3d_ve_perf",
                                            [31, 31, 31], "1 rank, nt=1, 201 PT iterations"),
    "test_Stokes3D_ve_perf.bson": ("scripts/stokes_3D/Stokes3D_ve_perf.jl", "3d_ve_perf", [31, 31, 31],
                                   "nt=1, 201 PT iterations"),
}


def _doc(b, off):
    size = struct.unpack_from("<i", b, off)[0]
    end = off + size
    off += 4
    out = {}
    while off < end - 1:
        t = b[off]
        off += 1
        z = b.index(b"\0", off)
        name = b[off:z].decode()
        off = z + 1
        if t == 0x01:
            v = struct.unpack_from("<d", b, off)[0]
            off += 8
        elif t == 0x02:
            n = struct.unpack_from("<i", b, off)[0]
            v = b[off + 4:off + 4 + n - 1].decode()
            off += 4 + n
        elif t in (0x03, 0x04):
            v, off = _doc(b, off)
            if t == 0x04:
                v = [v[k] for k in sorted(v, key=int)]
        elif t == 0x05:
            n = struct.unpack_from("<i", b, off)[0]
            v = bytes(b[off + 5:off + 5 + n])
            off += 5 + n
        elif t == 0x08:
            v = bool(b[off])
            off += 1
        elif t == 0x10:
            v = struct.unpack_from("<i", b, off)[0]
            off += 4
        elif t == 0x12:
            v = struct.unpack_from("<q", b, off)[0]
            off += 8
        elif t == 0x0A:
            v = None
        else:
            raise ValueError(f"unsupported BSON element type {t:#x}")
        out[name] = v
    return out, end


def _array(d):
    assert d["tag"] == "array" and d["type"]["name"] == ["Core", "Float64"], d.get("type")
    size = [int(s) for s in d["size"]]
    n = 1
    for s in size:
        n *= s
    vals = struct.unpack(f"<{n}d", d["data"])
    return {"size": size, "order": "column-major", "hex": [float(v).hex() for v in vals]}


def main(ref_root):
    src = os.path.join(ref_root, "test", "reftest-files")
    for name, (script, variant, grid, run) in RUNS.items():
        raw = open(os.path.join(src, name), "rb").read()
        doc, _ = _doc(raw, 0)
        out = {
            "source": f"test/reftest-files/{name}",
            "source_md5": hashlib.md5(raw).hexdigest(),
            "script": script,
            "variant": variant,
            "grid": grid,
            "run": run,
            "compare": "isapprox on each array: norm(a-b) <= sqrt(eps(Float64))*max(norm(a),norm(b))",
            "P": _array(doc["P"]),
            "X": _array(doc["X"]),
        }
        dst = os.path.join(HERE, name.replace(".bson", ".json"))
        with open(dst, "w") as fh:
            json.dump(out, fh, indent=0)
        print("wrote", dst)


def reference_dir():
    """The reference checkout: the first argument, else $PTS_REFERENCE_DIR."""
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PTS_REFERENCE_DIR")
    if not ref:
        sys.exit("usage: python tests/golden/make_golden.py /path/to/reference  (or set PTS_REFERENCE_DIR)")
    return ref


if __name__ == "__main__":
    main(reference_dir())
