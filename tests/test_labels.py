"""Island labelling: the oracle pinned to the reference's label propagation
and known answers (CPU), and the GPU union-find bit-exact against it.

Reference behaviour restated:
  * labels are the fixed point of hook-to-min / pointer-jump propagation
    from label i + 1 (SH/label_prop_init.comp.glsl, label_prop_iterate.comp.glsl;
    PFSFLabelPropCpuSimulator.java), i.e. 1 + the smallest flat index of each
    26-connected component; air 0xFFFFFFFF;
  * component records {root, count, anchored, aabb} agree with a rescan
    (GpuLabelPropSimulatorTest.java:94-137); more than 64 components set the
    overflow flag and clamp the count (:164-207);
  * random domains 4..10 per side, 55 % solid / 10 % anchor
    (GpuLabelPropSimulatorTest.java:40-90);
  * a 5x5x5 cluster floating over an anchored floor: 125 orphans; one solid
    voxel bridging it to the floor: 0 (validation/FloatingIslandTest.java:26-115).
"""
import numpy as np
import pytest

import oracle as O

NO = 0xFFFFFFFF


def _random_domain(rng, lo=4, hi=10):
    dims = tuple(int(v) for v in rng.integers(lo, hi + 1, 3))
    r = rng.random(int(np.prod(dims)))
    vt = np.where(r < 0.55, 1, np.where(r < 0.65, 2, 0)).astype(np.uint8)
    return dims, vt


def _rescan(dims, vt, labels):
    lx, ly, lz = dims
    out = {}
    for i in np.where(labels != NO)[0]:
        x, y, z = i % lx, (i // lx) % ly, i // (lx * ly)
        c = out.setdefault(int(labels[i]), [0, 0, [NO] * 3, [0] * 3])
        c[0] += 1
        c[1] |= int(vt[i] == 2)
        for a, v in enumerate((x, y, z)):
            c[2][a] = min(c[2][a], int(v))
            c[3][a] = max(c[3][a], int(v))
    return [[k, v[0], v[1], 0, *v[2], 0, *v[3], 0] for k, v in sorted(out.items())]


def floating_island(with_bridge=False):
    L, g = 11, 5
    vt = np.zeros(L ** 3, np.uint8)
    vt[: L * L] = 2  # z = 0 floor of anchors
    o = (L - g) // 2
    for z in range(2, 2 + g):
        for y in range(o, o + g):
            for x in range(o, o + g):
                vt[x + L * (y + L * z)] = 1
    if with_bridge:
        vt[L // 2 + L * (L // 2 + L * 1)] = 1
    return (L, L, L), vt


def orphans(dims, vt, labels, comps):
    anchored = {int(c[0]) for c in comps if c[2]}
    return int(np.sum((vt == 1) & ~np.isin(labels, list(anchored))))


def test_oracle_is_the_label_propagation_fixed_point():
    rng = np.random.default_rng(20260101)
    for _ in range(100):
        dims, vt = _random_domain(rng)
        lab, comps, cnt = O.label_components(dims, vt, cap=10 ** 6)
        lp, _ = O.label_propagation(dims, vt)
        np.testing.assert_array_equal(lab, lp)
        assert comps.tolist() == _rescan(dims, vt, lab)
        assert cnt == len(comps)


def test_oracle_overflow_and_orphans():
    L = 10
    vt = np.zeros(L ** 3, np.uint8)
    cnt = 0
    for z in range(0, L, 2):
        for y in range(0, L, 2):
            for x in range(0, L, 2):
                if cnt < 72:
                    vt[x + L * (y + L * z)] = 1
                    cnt += 1
    lab, comps, n = O.label_components((L, L, L), vt, cap=64)
    assert n == 72 and len(comps) == 64
    dims, vt = floating_island()
    lab, comps, n = O.label_components(dims, vt, cap=64)
    assert orphans(dims, vt, lab, comps) == 125
    dims, vt = floating_island(with_bridge=True)
    lab, comps, n = O.label_components(dims, vt, cap=64)
    assert orphans(dims, vt, lab, comps) == 0 and n == 1


@pytest.fixture(scope="module")
def eng(lib_built):
    from pfsf_b200 import capi
    e = capi.Engine(capi.default_config(max_island_size=1 << 26, tick_budget_ms=1 << 30))
    assert e.init() == capi.PFSF_OK, "CUDA device required"
    yield e
    e.close()


@pytest.mark.gpu
def test_gpu_labels_random_domains(eng):
    rng = np.random.default_rng(20260101)
    for _ in range(100):
        dims, vt = _random_domain(rng)
        rc, lab, comps, cnt, ovf = eng.label_components(vt, dims, capacity=4096)
        want, wcomps, wcnt = O.label_components(dims, vt, cap=4096)
        assert rc == 0
        np.testing.assert_array_equal(lab, want)
        np.testing.assert_array_equal(comps, wcomps)
        assert cnt == wcnt and ovf == 0


@pytest.mark.gpu
def test_gpu_labels_known_answers(eng):
    L = 10
    vt = np.zeros(L ** 3, np.uint8)
    cnt = 0
    for z in range(0, L, 2):
        for y in range(0, L, 2):
            for x in range(0, L, 2):
                if cnt < 72:
                    vt[x + L * (y + L * z)] = 1
                    cnt += 1
    rc, lab, comps, n, ovf = eng.label_components(vt, (L, L, L), capacity=64)
    assert rc == 0 and n == 64 and ovf == 1
    for bridge, want in ((False, 125), (True, 0)):
        dims, vt = floating_island(bridge)
        rc, lab, comps, n, ovf = eng.label_components(vt, dims)
        assert rc == 0 and orphans(dims, vt, lab, comps) == want
    # empty and all-air boxes
    rc, lab, comps, n, ovf = eng.label_components(np.zeros(27, np.uint8), (3, 3, 3))
    assert rc == 0 and n == 0 and np.all(lab == NO)
    # components only, no label array
    dims, vt = floating_island()
    rc, lab, comps, n, ovf = eng.label_components(vt, dims, labels=False)
    assert rc == 0 and lab is None and n == 2


@pytest.mark.gpu
def test_gpu_labels_large_noise_domains(eng):
    """Big boxes with long, thin components (value noise thresholded near
    the percolation point) -- many unions per root."""
    from pfsf_b200 import synth
    for dims, seed, occ in (((256, 128, 96), 3, 0.35), ((97, 61, 203), 5, 0.5), ((512, 8, 8), 7, 0.3)):
        rng = np.random.default_rng(seed)
        noise = synth._value_noise(dims, rng)
        thr = np.quantile(noise, 1 - occ)
        vt = (noise > thr).astype(np.uint8).reshape(-1)
        vt[(rng.random(vt.size) < 0.02) & (vt == 1)] = 2
        rc, lab, comps, n, ovf = eng.label_components(vt, dims, capacity=1 << 16)
        want, wcomps, wn = O.label_components(dims, vt, cap=1 << 16)
        assert rc == 0
        np.testing.assert_array_equal(lab, want)
        np.testing.assert_array_equal(comps, wcomps)
        assert n == min(wn, 1 << 16)
