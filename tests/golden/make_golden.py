"""Regenerates the golden fixtures in this directory from the reference
checkout. Run once in a container that has the reference; the outputs are
committed and nothing at test time reads the reference.

  python tests/golden/make_golden.py [--ref /path/to/exahype]

Writes
  kernel_vectors.npz  every array of the reference's kernel-test data files
                      (ExaHyPE/exahype/tests/kernels/testdata/
                      {generic_euler,limiter,elasticity}_testdata.cpp), read
                      as text and keyed "<dim>/<file>/<namespace>/<array>".
  ref_tables.npz      the reference's operator tables, dumped by its own init
                      code compiled into oracle/_ref (key "<name>/<N>").
  ref_mesh_*.npz      uniform-mesh runs of the reference kernels through the
                      oracle harness (see tests/test_oracle_ref.py for what
                      each holds); generated only when oracle/_ref is built.
"""
import argparse
import ctypes
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))

ARRAY_RE = re.compile(r"const\s+double\s+(\w+)\s*\[\s*([\d\s*]+?)\s*\]\s*=?\s*\{(.*?)\}\s*;", re.S)


def parse_testdata(path):
    """Maps '<dim>/<namespace>/<name>' -> float64 array for every initialised
    `const double name[n] = {...};` in a reference test-data file."""
    text = open(path).read()
    text = re.sub(r"//[^\n]*", "", text)
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    out = {}
    # split into Dim2 / Dim3 sections
    for dim_tag, dim in (("Dim2", "2d"), ("Dim3", "3d")):
        m = re.search(r"#ifdef\s+%s(.*?)#endif" % dim_tag, text, re.S)
        if not m:
            continue
        sec = m.group(1)
        # walk namespaces in order
        pos = 0
        ns = None
        for tok in re.finditer(r"namespace\s+(\w+)\s*\{|const\s+double\s+\w+\s*\[", sec):
            if tok.group(0).startswith("namespace"):
                ns = tok.group(1)
                continue
            am = ARRAY_RE.match(sec, tok.start())
            if not am:
                continue
            name, body = am.group(1), am.group(3)
            n = int(np.prod([int(f) for f in am.group(2).split("*")]))  # sizes like "9 * 5 * 4"
            vals = [float(v) for v in re.split(r"[,\s]+", body.strip()) if v]
            if not vals:
                continue
            arr = np.zeros(n)
            arr[: len(vals)] = vals
            out["%s/%s/%s" % (dim, ns, name)] = arr
    return out


def make_kernel_vectors(ref):
    td = os.path.join(ref, "ExaHyPE", "exahype", "tests", "kernels", "testdata")
    out = {}
    for fname in ("generic_euler_testdata.cpp", "limiter_testdata.cpp", "elasticity_testdata.cpp"):
        for k, v in parse_testdata(os.path.join(td, fname)).items():
            dim, rest = k.split("/", 1)
            out["%s/%s/%s" % (dim, fname.split("_testdata")[0], rest)] = v
    np.savez_compressed(os.path.join(HERE, "kernel_vectors.npz"), **out)
    return out


def make_ref_tables():
    lib = ctypes.CDLL(os.path.join(REPO, "oracle", "_ref", "libexaref2d.so"))
    buf = (ctypes.c_double * 512)()
    out = {}
    for name in ("nodes", "weights", "lobatto_nodes", "lobatto_weights", "FLCoeff", "FRCoeff", "FCoeff", "Kxi",
                 "iK1", "dudx", "uh2lim", "lim2uh", "uh2lob", "fineGridProjector1d", "equidistantGridProjector1d"):
        for N in range(1, 10):
            n = lib.ref2d_table(name.encode(), N, buf)
            out["%s/%d" % (name, N)] = np.array(buf[:n])
    np.savez_compressed(os.path.join(HERE, "ref_tables.npz"), **out)
    return out


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=None, help="reference checkout (default: $EXAHYPE_REFERENCE, else a "
                    "directory named 'reference' beside this repository)")
    a = ap.parse_args()
    if a.ref is None:
        sys.path.insert(0, os.path.join(REPO, "oracle"))
        import pyoracle
        a.ref = pyoracle.reference_root()
        assert a.ref, "no reference checkout found"
    kv = make_kernel_vectors(a.ref)
    print("kernel_vectors: %d arrays" % len(kv))
    if os.path.exists(os.path.join(REPO, "oracle", "_ref", "libexaref2d.so")):
        rt = make_ref_tables()
        print("ref_tables: %d arrays" % len(rt))
        sys.path.insert(0, HERE)
        try:
            import make_ref_mesh  # noqa: F401  (optional: mesh-run fixtures)
            make_ref_mesh.main()
        except ImportError:
            pass
