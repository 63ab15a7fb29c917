"""Output kernels against the reference: the XZ plane dump (savePlaneXZ,
ComputeUnitOutput.hpp:354-447) read back from the reference's own files,
and the vorticity slices (calcVorticityXZ/XY, :113-285) against the
reference's expression evaluated on its own moments.

Stated tolerances: record coordinates and counts exact; moments and F of
the records within the step tolerance of the parity tests (2e-6 per step
relative L2, F 5e-5); log |curl u|^2 within 1e-2 where |curl u|^2 > 1e-9
(central differences of nearly equal velocities lose relative precision).
"""
import os

import numpy as np
import pytest

from test_gpu_parity import random_markers, rel_l2

pytestmark = pytest.mark.gpu

ALPHA, BETA = 0.97, 1.9
DIMS = (14, 12, 16)
STEPS = 4


def run_pair(tb, po, tmp, streaming="Simple"):
    x, y, z = DIMS
    rng = np.random.default_rng(77)
    flow = po.Flow(initialRho=1.0, nu=2e-3, cs0=0.1, g3=0.8, alpha=ALPHA, beta=BETA, useLES=True)
    lat = po.CpuLattice("ref", x, y, z, flow, streaming, 4, tmpdir=str(tmp))
    cu = tb.ComputeUnit(x=x, y=y, z=z, nu=2e-3, cs0=0.1, g3=0.8, useLES=1, initialRho=1.0,
                        streaming=tb.STREAMING_SIMPLE if streaming == "Simple" else tb.STREAMING_ESOTWIST)
    mks = [random_markers(tb, rng, x * z // 2, x, y, z, planes=[2, y // 2, y - 3]) for _ in range(STEPS + 1)]
    lat.initialise(1.0)
    cu.initialise(1.0)
    lat.forcing(mks[0], ALPHA, BETA)
    cu.forcing(mks[0], ALPHA, BETA)
    for mk in mks[1:]:
        lat.step(mk, ALPHA, BETA)
        cu.collision()
        cu.forcing(mk, ALPHA, BETA)
    return cu, lat, mks[-1]


@pytest.mark.parametrize("streaming", ["Simple", "Esotwist"])
def test_plane_xz_matches_reference_files(gpu, ref_oracle, tmp_path, streaming):
    tb, po = gpu, ref_oracle
    cu, lat, mk = run_pair(tb, po, tmp_path, streaming)
    excl = mk[: len(mk) // 3]
    cu.set_output_exclude(excl)
    lat.set_exclude(excl)
    j = DIMS[1] // 2                       # a plane with markers
    q, f = cu.plane_xz(j)
    d = lat.save_plane_xz(j + 1, 5)        # the reference's j counts the ghost layer
    rq = np.fromfile(os.path.join(d, "CUid.0.0.0.V5.QVec.bin"), tb.DISK_GRID4_DTYPE)
    rf = np.fromfile(os.path.join(d, "CUid.0.0.0.V5.F3.bin"), tb.DISK_GRID3_DTYPE)
    assert len(q) == len(rq) and len(q) < DIMS[0] * DIMS[2]
    for c in ("iGrid", "jGrid", "kGrid"):
        np.testing.assert_array_equal(q[c], rq[c])
        np.testing.assert_array_equal(f[c], rf[c])
    assert len(f) > 0
    assert rel_l2(q["q"][:, 0], rq["q"][:, 0]) <= 2e-6 * STEPS
    assert rel_l2(q["q"][:, 1:], rq["q"][:, 1:]) <= 5e-5
    assert rel_l2(f["q"], rf["q"]) <= 5e-5
    cu.set_output_exclude(excl, False)
    q2, _ = cu.plane_xz(j)
    assert len(q2) == DIMS[0] * DIMS[2]
    cu.close()


def curl_log(m, axis, cut):
    """The reference's vorticity expression on moments m[x, y, z, >=4],
    interior neighbours only (cells next to a lattice face are NaN)."""
    u = m[..., 1:4] / m[..., :1]
    x, y, z = u.shape[:3]
    out = np.full((x, z) if axis == "xz" else (y, x), np.nan)
    for i in range(1, x - 1):
        for b in range(1, (z if axis == "xz" else y) - 1):
            j, k = (cut, b) if axis == "xz" else (b, cut)
            if not (0 < j < y - 1 and 0 < k < z - 1):
                continue
            uxy = 0.5 * (u[i, j, k + 1, 0] - u[i, j, k - 1, 0])
            uxz = 0.5 * (u[i, j + 1, k, 0] - u[i, j - 1, k, 0])
            uyx = 0.5 * (u[i + 1, j, k, 1] - u[i - 1, j, k, 1])
            uyz = 0.5 * (u[i, j + 1, k, 1] - u[i, j - 1, k, 1])
            uzx = 0.5 * (u[i + 1, j, k, 2] - u[i - 1, j, k, 2])
            uzy = 0.5 * (u[i, j, k + 1, 2] - u[i, j, k - 1, 2])
            v = (uyz - uzy) ** 2 + (uzx - uxz) ** 2 + (uxy - uyx) ** 2
            if axis == "xz":
                out[i, k] = np.log(v) if v > 0 else -np.inf
            else:
                out[j, i] = np.log(v) if v > 0 else -np.inf
    return out


@pytest.mark.parametrize("streaming", ["Simple", "Esotwist"])
def test_vorticity_slices_match_reference_expression(gpu, ref_oracle, tmp_path, streaming):
    tb, po = gpu, ref_oracle
    cu, lat, mk = run_pair(tb, po, tmp_path, streaming)
    m = lat.get_moments()
    for axis, cut in (("xz", DIMS[1] // 2), ("xy", DIMS[2] // 2)):
        got = cu.vorticity_xz(cut) if axis == "xz" else cu.vorticity_xy(cut)
        want = curl_log(m, axis, cut)
        ok = np.isfinite(want) & (want > np.log(1e-9))
        assert ok.sum() > 20
        assert np.max(np.abs(got[ok] - want[ok])) <= 1e-2
    cu.set_output_exclude(mk)
    got = cu.vorticity_xz(DIMS[1] // 2)
    sel = mk[mk["j"] == DIMS[1] // 2]
    assert np.all(got[sel["i"], sel["k"]] == -1.0)
    cu.close()
