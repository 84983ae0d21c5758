"""Generates the committed golden vectors under tests/golden/.

    python tests/golden/make_golden.py [--reference /path/to/PFSF-CORE]

fixtures_compat.npz -- the reference's 21 schema-v1 fixtures
    (Block Reality/api/src/test/resources/pfsf-fixtures/*.json, inputs only:
    dims, material ids, registry, anchors, wind) converted to tick inputs with
    the reference data-assembly rules (tests/cases.py load_fixture).  Read from
    the reference checkout when it is present; the GPU box has no checkout,
    so the converted arrays are committed.
golden_ticks.npz -- oracle outputs (phi after each of 3 ticks, failure
    flags, H, damage, schedule state) for small synthetic cases, so a change
    to the oracle shows up as a diff against these vectors.
"""
import argparse
import glob
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, "tests"), os.path.join(ROOT, "oracle"), os.path.join(ROOT, "pfsf-core_b200")]

import cases  # noqa: E402
import oracle as O  # noqa: E402

FIELDS = ("phi", "source", "conductivity", "type", "rcomp", "rtens", "max_phi", "hydration")


def fixtures(ref_root):
    pat = os.path.join(ref_root, "Block Reality", "api", "src", "test", "resources", "pfsf-fixtures", "*.json")
    out = {}
    for path in sorted(glob.glob(pat)):
        c = cases.load_fixture(path)
        nm = os.path.splitext(os.path.basename(path))[0]
        out[f"{nm}__dims"] = np.array(c["dims"], np.int32)
        for f in FIELDS:
            out[f"{nm}__{f}"] = c[f]
    return out


def ticks():
    out = {}
    for nm in ("block8", "noise20", "rod"):
        c = cases.compat_case(nm)
        I = O.Island(*c["dims"])
        I.load(**{f: c[f] for f in FIELDS})
        out[f"{nm}__dims"] = np.array(c["dims"], np.int32)
        for f in FIELDS:
            out[f"{nm}__in_{f}"] = c[f]
        for t in range(3):
            I.tick()
            out[f"{nm}__phi_t{t}"] = I.view("phi").copy()
        out[f"{nm}__fail"] = I.view("fail").astype(np.uint8)
        out[f"{nm}__H"] = I.view("H").copy()
        out[f"{nm}__D"] = I.view("D").copy()
        st = I.state()
        out[f"{nm}__state"] = np.array([st["chebyshev_iter"], st["pcg_allocated"], st["mg_allocated"]], np.int32)
    return out


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("PFSF_REFERENCE", os.path.join(os.path.dirname(ROOT), "reference")),
                    help="reference checkout (default: $PFSF_REFERENCE, else ../reference beside this repository)")
    a = ap.parse_args()
    if os.path.isdir(a.reference):
        fx = fixtures(a.reference)
        np.savez_compressed(os.path.join(HERE, "fixtures_compat.npz"), **fx)
        print("fixtures:", len({k.split('__')[0] for k in fx}))
    np.savez_compressed(os.path.join(HERE, "golden_ticks.npz"), **ticks())
    print("golden ticks written")
