"""Pins the CPU restatement (oracle/tdlb_oracle.c) to the reference.

1. The reference's own golden streaming vectors
   (tdlbcpp/tests/StreamingSimplePushTest.hpp, StreamingSimpleTest.hpp) equal
   both the reference compiled in place and the restatement.
2. The restatement's integer-coded transport (Simple push/pull, Esotwist
   read/write/writeMoments maps) equals the reference's AccessField code.
3. Full time steps (collision, streaming, moments, IBM forcing with
   overlapping markers) are bit-identical between restatement and reference
   in FP32 and FP64, LES on and off, Simple and Esotwist.
"""
import numpy as np
import pytest


def random_markers(po, rng, n, x, y, z):
    m = np.zeros(n, po.MARKER_DTYPE)
    m["i"] = rng.integers(0, x, n)
    m["j"] = rng.integers(0, y, n)
    m["k"] = rng.integers(0, z, n)
    m["iCartFraction"] = rng.uniform(-0.5, 0.5, n)
    m["kCartFraction"] = rng.uniform(-0.5, 0.5, n)
    m["uDelta"] = rng.uniform(-0.1, 0.1, n)
    m["vDelta"] = rng.uniform(-0.1, 0.1, n)
    m["wDelta"] = rng.uniform(-0.1, 0.1, n)
    return m


@pytest.mark.parametrize("push", [True, False])
def test_golden_streaming_vectors(ref_oracle, port_oracle, push):
    po = ref_oracle
    golden = po.kat_simple_golden(push)
    assert golden.shape == (5, 5, 5, 18)
    np.testing.assert_array_equal(po.kat_simple_stream("ref", push, 3, 3, 3), golden)
    np.testing.assert_array_equal(po.kat_simple_stream("port", push, 3, 3, 3), golden)


@pytest.mark.parametrize("dims", [(3, 3, 3), (4, 5, 6), (7, 3, 5), (1, 2, 3)])
def test_simple_push_matches_reference(ref_oracle, port_oracle, dims):
    po = ref_oracle
    for push in (True, False):
        np.testing.assert_array_equal(po.kat_simple_stream("port", push, *dims), po.kat_simple_stream("ref", push, *dims))


@pytest.mark.parametrize("dims", [(3, 3, 3), (4, 5, 6), (7, 3, 5), (2, 2, 2)])
def test_esotwist_maps_match_reference(ref_oracle, port_oracle, dims):
    po = ref_oracle
    for even in (True, False):
        np.testing.assert_array_equal(po.kat_esotwist_read("port", *dims, even), po.kat_esotwist_read("ref", *dims, even))
        for moments_map in (False, True):
            for n in (1, 2, 3):
                np.testing.assert_array_equal(po.kat_esotwist("port", *dims, even, n, moments_map),
                                              po.kat_esotwist("ref", *dims, even, n, moments_map))


def test_esotwist_is_periodic_streaming(port_oracle):
    """An even read + write, then the odd read, moves every population by its
    lattice vector with periodic wrap over the interior."""
    po = port_oracle
    x, y, z = 4, 5, 6
    state = po.kat_esotwist("port", x, y, z, True, 1, False)
    # after one even write + flip, the odd read map yields the streamed values
    lat = po.CpuLattice("port", x, y, z, po.Flow(), "Esotwist", 8)
    lat.set_q(state.astype(np.float64))
    lat.even_step = False
    got = lat.get_moments()
    from tdlbcpp_b200 import CX, CY, CZ
    want = np.empty_like(got)
    first = po.kat_esotwist_read("port", x, y, z, True).astype(np.float64)   # what the even step read
    for d in range(18):
        want[..., d] = np.roll(first[..., d], shift=(CX[d], CY[d], CZ[d]), axis=(0, 1, 2))
    np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize("streaming", ["Simple", "Esotwist"])
@pytest.mark.parametrize("precision", [4, 8])
@pytest.mark.parametrize("les", [True, False])
def test_restatement_bit_identical(ref_oracle, port_oracle, streaming, precision, les):
    po = ref_oracle
    rng = np.random.default_rng(1234 + precision + 2 * les)
    x, y, z = 9, 7, 11
    flow = po.Flow(initialRho=1.0, nu=2e-3, cs0=0.1, g3=0.8, useLES=les)
    lats = [po.CpuLattice(k, x, y, z, flow, streaming, precision) for k in ("port", "ref")]
    mk = random_markers(po, rng, 150, x, y, z)
    for L in lats:
        L.initialise(1.0)
        L.forcing(mk, 0.97, 1.9)
    for _ in range(5):
        mk = random_markers(po, rng, 150, x, y, z)
        for L in lats:
            L.step(mk, 0.97, 1.9)
    a, b = lats
    np.testing.assert_array_equal(a.get_moments(), b.get_moments())
    np.testing.assert_array_equal(a.interior(a.get_f()), b.interior(b.get_f()))
    np.testing.assert_array_equal(a.interior(a.get_nu()), b.interior(b.get_nu()))
    assert a.even_step == b.even_step


@pytest.mark.parametrize("re,uav,radius", [(7300.0, 0.1, 10), (20000.0, 0.1, 66), (1276.9886727287553, 0.1, 8),
                                           (13432.792223087894, 0.07532754608704051, 21)])
def test_nu_from_reynolds_bit_exact_with_reference(ref_oracle, re, uav, radius):
    """The host's calcNuAndRe_m restatements equal the reference's own."""
    import tdlbcpp_b200 as tb
    lib = ref_oracle.load("ref")
    assert tb.nu_from_reynolds(re, uav, radius) == lib.tdlbref_calc_nu(re, uav, radius)


@pytest.mark.parametrize("edge", [16, 60, 400])
def test_reference_harness_geometry_equals_product_generator(ref_oracle, edge):
    """The marker generator compiled into the reference harness (used by
    bench.py's reference arm, which must not load the B200 library) gives the
    product generator's lists bit for bit, and the reference's own
    calcNuAndRe_m gives the product's nu."""
    import tdlbcpp_b200 as tb
    po = ref_oracle
    a = po.RefRushton(edge, edge, edge, tip_speed=0.1)
    b = tb.RushtonTurbine(edge, edge, edge, tip_speed=0.1)
    d = a.increment(1)
    assert d == b.increment(1) and a.blade_outer_radius() == b.blade_outer_radius()
    for angle in (0.0, 0.37, 2.5):
        assert a.forcing_list(angle, d).tobytes() == b.forcing_list(angle, d).tobytes()
    assert po.ref_nu(20000.0, 0.1, a.blade_outer_radius()) == tb.nu_from_reynolds(20000.0, 0.1, b.blade_outer_radius())


@pytest.mark.parametrize("streaming", ["Simple", "Esotwist"])
def test_restatement_bit_identical_on_400_cubed_slab(ref_oracle, port_oracle, streaming):
    """Ties the restatement to the reference at the at-scale geometry: a
    400 x 16 x 400 slab through the impeller plane of the 400^3 tank (Re
    20000, tip speed 0.1, LES, the slab's markers of the project generator),
    forcing plus two time steps, FP32: moments, F and Nu bit for bit."""
    po = ref_oracle
    edge, height = 400, 16
    rt = po.RefRushton(edge, edge, edge, tip_speed=0.1)
    nu = po.ref_nu(20000.0, 0.1, rt.blade_outer_radius())
    dth = rt.increment(1)
    j0 = int(round(edge / 3.0)) - height // 2

    def slab(angle):
        m = rt.forcing_list(angle, dth, nonupdating_delta=dth)
        m = m[(m["j"] >= j0) & (m["j"] < j0 + height)].copy()
        m["j"] -= j0
        return m

    flow = po.Flow(initialRho=1.0, nu=nu, cs0=0.1, g3=0.8, useLES=True)
    lats = [po.CpuLattice(k, edge, height, edge, flow, streaming, 4) for k in ("port", "ref")]
    mk = slab(0.0)
    assert len(mk) > 1000
    for L in lats:
        L.initialise(1.0)
        L.forcing(mk, 0.97, 1.9)
    angle = 0.0
    for _ in range(2):
        angle += dth
        mk = slab(angle)
        for L in lats:
            L.step(mk, 0.97, 1.9)
    a, b = lats
    np.testing.assert_array_equal(a.get_moments(), b.get_moments())
    np.testing.assert_array_equal(a.interior(a.get_f()), b.interior(b.get_f()))
    np.testing.assert_array_equal(a.interior(a.get_nu()), b.interior(b.get_nu()))
    for L in lats:
        L.close()
