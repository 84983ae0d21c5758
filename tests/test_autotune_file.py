"""The tuning file the autotuner writes: one section per GPU, rewritten in
place, read back by the same rules the engine uses (no GPU needed)."""
from pfsf_b200 import autotune

P = {"cluster": 4, "cluster_min_voxels": 262144, "grid_min_voxels": 2097152, "warp_max_voxels": 0, "cheb_k": 3,
     "cheb_lower": 0.15, "coarse_weight": 1.6, "tail_cells": 128, "coarse_sweeps": 3, "inner_eta": 0.0003}


def _read(path):
    out, cur = {}, None
    for ln in open(path).read().splitlines():
        s = ln.strip()
        if not s or s.startswith("#"):
            continue
        if s.startswith("[") and s.endswith("]"):
            cur = s[1:-1].strip()
            out[cur] = {}
            continue
        k, v = (x.strip() for x in s.split("=", 1))
        out[cur][k] = float(v) if k in autotune.FLOAT_KEYS else int(v)
    return out


def test_sections_are_written_and_replaced(tmp_path):
    path = str(tmp_path / "t" / "pfsf_tune.txt")
    autotune.write_section(path, "GPU A 148", P, note="first")
    autotune.write_section(path, "GPU B 132", dict(P, cluster=8))
    autotune.write_section(path, "GPU A 148", dict(P, cheb_k=2), note="again")
    got = _read(path)
    assert set(got) == {"GPU A 148", "GPU B 132"}
    assert got["GPU A 148"] == dict(P, cheb_k=2)
    assert got["GPU B 132"]["cluster"] == 8
