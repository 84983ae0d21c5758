"""pfsf_tick_tolerance: the reference tick with its fixed schedule replaced by
the tolerance solve, against the oracle.

Per tick (load ramped between ticks, warm start from the previous phi):
  * phi: FP64-evaluated relative residual <= 1e-6, the FP32 phi is the FP64
    accumulator rounded, error vs the oracle's FP64 solve <= 1e-4;
  * on that phi, the oracle's history update, phase field and failure scan
    (oracle.tolerance_tick_tail): failure flags and the failure buffer
    (count and every {x,y,z,type} tuple) bit-exact, H and damage within 1e-5
    of their maxima -- the tolerances of the reference-schedule parity tests.
"""
import numpy as np
import pytest

import oracle as O
from pfsf_b200 import capi, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng(lib_built):
    e = capi.Engine(capi.default_config(max_island_size=1 << 26, tick_budget_ms=1 << 30))
    assert e.init() == capi.PFSF_OK, "CUDA device required"
    yield e
    e.close()


def _case(dims, seed, phi_max=20.0, rscale=0.1):
    isl = synth.noise_island(dims, seed=seed)
    phi, _, _ = O.kappa_solve64(isl.dims, isl.kappa.astype(np.float64), isl.vtype, isl.source.astype(np.float64),
                                tol=1e-10)
    scale = phi_max / np.abs(phi).max()  # loads scaled so the phase field and the scan act
    case = {"conductivity": synth.face_sigma_from_kappa(isl.dims, isl.vtype, isl.kappa),
            "type": isl.vtype.copy(), "rcomp": (isl.rcomp * rscale).astype(np.float32),
            "rtens": (isl.rtens * rscale).astype(np.float32), "max_phi": np.full(isl.n, 1e9, np.float32),
            "hydration": np.ones(isl.n, np.float32), "source": (isl.source * scale).astype(np.float32)}
    return isl, case


@pytest.mark.parametrize("prec", [capi.PREC_BF16, capi.PREC_FP32])
def test_tick_tolerance_matches_oracle(eng, prec):
    eng.set_solve_mode(capi.SOLVE_BATCHED)
    eng.set_precision(prec)
    cases = [_case((24, 20, 16), 12), _case((17, 13, 11), 13, rscale=0.3)]
    ids, hosts, refs = [], [], []
    for k, (isl, case) in enumerate(cases):
        iid = 9100 + 10 * prec + k
        origin = (5 * k, -3, 2)
        assert eng.add_island(iid, isl.dims, origin) == capi.PFSF_OK
        h = {"phi": np.zeros(isl.n, np.float32), "phik": np.zeros(isl.n, np.float32),
             "source": case["source"].copy(), "base": case["source"].copy()}
        assert eng.register_buffers(iid, h["phi"], h["source"], case["conductivity"], case["type"], case["rcomp"],
                                    case["rtens"], case["max_phi"]) == capi.PFSF_OK
        assert eng.register_kappa(iid, h["phik"], h["source"], isl.kappa, isl.vtype) == capi.PFSF_OK
        ids.append(iid)
        hosts.append(h)
        refs.append({"H": np.zeros(isl.n, np.float32), "D": np.zeros(isl.n, np.float32),
                     "fail": np.zeros(isl.n, np.uint32), "origin": origin})
    cap = 8192
    saw_fail = False
    for t in range(3):
        f = 1.0 + 0.5 * t
        for h in hosts:
            h["source"][:] = h["base"] * np.float32(f)
        for iid in ids:  # the Java runtime marks its islands dirty every tick
            eng.L.pfsf_mark_full_rebuild(eng.h, iid)
        fb = np.zeros(1 + 4 * cap, np.int32)
        fb[0] = 99
        rc, st = eng.tick_tolerance(ids, fb, tol=1e-6)
        assert rc == capi.PFSF_OK and st.islands_converged == len(ids), st.max_rel_residual
        want = np.zeros(1 + 4 * cap, np.int32)
        for (isl, case), iid, h, r in zip(cases, ids, hosts, refs):
            rc, x64 = eng.read_solution64(iid, isl.n)
            np.testing.assert_array_equal(h["phik"], x64.astype(np.float32))
            k64 = isl.kappa.astype(np.float64)
            s64 = h["source"].astype(np.float64)
            res = s64 - O.kappa_apply(isl.dims, k64, isl.vtype, x64)
            sol = isl.vtype == 1
            assert np.linalg.norm(res[sol]) <= 1e-6 * np.linalg.norm(s64[sol])
            xr, _, _ = O.kappa_solve64(isl.dims, k64, isl.vtype, s64, tol=1e-12)
            assert np.abs(x64 - xr).max() <= 1e-4 * np.abs(xr).max()
            c = dict(case, source=h["source"])
            O.tolerance_tick_tail(isl.dims, h["phik"], c, r["H"], r["D"], r["fail"])
            assert np.array_equal(eng.debug_field(iid, 3), r["fail"].astype(np.uint8)), f"tick {t}: fail flags"
            for field, name in ((1, "H"), (2, "D")):
                g = eng.debug_field(iid, field)
                sc = max(float(np.abs(r[name]).max()), 1e-30)
                assert float(np.abs(g - r[name]).max()) / sc <= 1e-5, f"tick {t}: {name}"
            ref_isl = O.Island(*isl.dims)
            ref_isl.load(phi=h["phik"], source=h["source"], conductivity=case["conductivity"], type=case["type"],
                         rcomp=case["rcomp"], rtens=case["rtens"], max_phi=case["max_phi"],
                         hydration=case["hydration"])
            ref_isl.view("fail")[:] = r["fail"]
            ref_isl.failures(r["origin"], capacity=cap, dbb=want)
        assert fb[0] == want[0], (t, fb[0], want[0])
        assert np.array_equal(fb[: 1 + 4 * fb[0]], want[: 1 + 4 * want[0]]), f"tick {t}: failure tuples"
        saw_fail |= fb[0] > 0
    assert saw_fail


def test_tick_tolerance_argument_errors(eng):
    isl = synth.noise_island((8, 8, 6), seed=3)
    iid = 9200
    assert eng.add_island(iid, isl.dims) == capi.PFSF_OK
    phi = np.zeros(isl.n, np.float32)
    assert eng.register_kappa(iid, phi, isl.source, isl.kappa, isl.vtype) == capi.PFSF_OK
    # no reference-layout buffers registered
    rc, _ = eng.tick_tolerance([iid])
    assert rc == capi.PFSF_ERROR_INVALID_ARG
    rc, _ = eng.tick_tolerance([iid], tol=0.0)
    assert rc == capi.PFSF_ERROR_INVALID_ARG
    rc, _ = eng.tick_tolerance([])
    assert rc == capi.PFSF_OK
