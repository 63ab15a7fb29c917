"""The step kernels' L2 prefetch spans, checked on the CPU.

`prefetch_ahead` (tdlbcpp_b200/csrc/step_kernels.cuh) has every eighth CTA
of a full step launch issue one `cp.async.bulk.prefetch.L2` per population
plane (and one for Nu) over the tiles one wave of resident CTAs further
on. This file restates its span arithmetic and checks, for every
prefetching CTA of several lattices, cell-per-thread variants, storage
widths and wave sizes, that each span starts on a 16-byte boundary, has a
non-zero size that is a multiple of 16 bytes, and stays inside its plane's
allocation (every plane starts 16-byte aligned and holds a multiple of 64
elements) -- and that it covers every element the target tiles' threads
pull from that plane away from the walls and the periodic wrap. The
batched kernel's per-chunk prefetch (`prefetch_chunk`, csrc/batch.cu) takes
the same spans over one chunk and is checked the same way.
"""
import numpy as np
import pytest

ROW_PITCH = 16          # TDLB_ROW_PITCH (csrc/tdlb_common.cuh)
TILES = 8               # kPrefetchTiles
CX = [1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0]
CY = [0, 0, 1, -1, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 1, -1]
CZ = [0, 0, 0, 0, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, -1, 1, -1, 1]


def dims(nx, ny, nz):
    kp = (nz + ROW_PITCH - 1) // ROW_PITCH * ROW_PITCH
    plane = (nx * ny * kp + 63) // 64 * 64
    return kp, plane


def shift(d, nx, ny, kp, eso, even):
    rs = ny * kp
    if eso:
        sg = -1 if even else 1
        return (rs if sg * CX[d] > 0 else 0) + (kp if sg * CY[d] > 0 else 0)
    return -(CX[d] * rs + CY[d] * kp)


def spans(nx, ny, nz, V, es, ahead, eso, even):
    """Byte spans [lo, hi) relative to plane d's base, per prefetching CTA."""
    kp, plane = dims(nx, ny, nz)
    tile = 128 * V
    grid = (nx * ny * (kp // V) + 127) // 128
    b = np.arange(0, grid, TILES, dtype=np.int64)
    e0 = (b + ahead) * tile
    live = e0 < nx * ny * kp
    b, e0 = b[live], e0[live]
    e1 = e0 + TILES * tile
    out = {}
    for d in range(18):
        sh = shift(d, nx, ny, kp, eso, even)
        a = np.clip(e0 + sh - 1, 0, plane)
        z = np.clip(e1 + sh + 1, 0, plane)
        ok = a < z
        lo = (a * es) // 16 * 16
        hi = (z * es + 15) // 16 * 16
        out[d] = (b[ok], e0[ok], lo[ok], hi[ok], plane * es)
    return out


@pytest.mark.parametrize("shape", [(400, 400, 400), (96, 96, 96), (45, 38, 51), (17, 5, 3)])
@pytest.mark.parametrize("V,es", [(1, 4), (2, 4), (4, 4), (1, 2), (2, 2), (4, 2)])
@pytest.mark.parametrize("ahead", [1, 592, 888, 1184])
@pytest.mark.parametrize("eso,even", [(False, False), (True, True), (True, False)])
def test_prefetch_spans_in_bounds_and_aligned(shape, V, es, ahead, eso, even):
    nx, ny, nz = shape
    for d, (b, e0, lo, hi, limit) in spans(nx, ny, nz, V, es, ahead, eso, even).items():
        assert (lo % 16 == 0).all() and (hi % 16 == 0).all()
        assert (hi > lo).all()
        assert (lo >= 0).all() and (hi <= limit).all(), d
        assert (hi - lo < 2 ** 32).all()


@pytest.mark.parametrize("shape", [(96, 96, 96), (45, 38, 51)])
@pytest.mark.parametrize("V", [1, 2, 4])
@pytest.mark.parametrize("eso,even", [(False, False), (True, True), (True, False)])
def test_prefetch_spans_cover_the_pulls(shape, V, eso, even):
    nx, ny, nz = shape
    kp, plane = dims(nx, ny, nz)
    rs = ny * kp
    es = 2
    checked = 0
    for d, (b, e0, lo, hi, limit) in spans(nx, ny, nz, V, es, 8, eso, even).items():
        b, e0, lo, hi = b[::7], e0[::7], lo[::7], hi[::7]   # a sample of the prefetching CTAs
        # every element of their target tiles, as (i, j, k), away from walls and wraps
        e = (e0[:, None] + np.arange(TILES * 128 * V)[None, :]).ravel()
        lo_r = np.repeat(lo, TILES * 128 * V)
        hi_r = np.repeat(hi, TILES * 128 * V)
        i, rem = np.divmod(e, rs)
        j, k = np.divmod(rem, kp)
        inner = (i >= 1) & (i < nx - 1) & (j >= 1) & (j < ny - 1) & (k >= 1) & (k < nz - 1)
        if eso:
            sg = -1 if even else 1
            src = e + (rs if sg * CX[d] > 0 else 0) + (kp if sg * CY[d] > 0 else 0) + (1 if sg * CZ[d] > 0 else 0)
        else:
            src = e - (CX[d] * rs + CY[d] * kp + CZ[d])
        byte = src * es
        sel = inner
        assert ((byte[sel] >= lo_r[sel]) & (byte[sel] + es <= hi_r[sel])).all(), d
        checked += int(sel.sum())
    assert checked > 0


@pytest.mark.parametrize("shape", [(48, 48, 48), (33, 17, 29)])
@pytest.mark.parametrize("V,NT", [(1, 128), (2, 128), (2, 256), (4, 256)])
@pytest.mark.parametrize("es", [2, 4])
@pytest.mark.parametrize("eso,even", [(False, False), (True, True), (True, False)])
def test_batched_chunk_spans_in_bounds_and_aligned(shape, V, NT, es, eso, even):
    """`prefetch_chunk` (csrc/batch.cu): the chunk of NT quads from quad q0,
    for every chunk start a block can prefetch (every multiple of NT up to
    the tank's quads, and the ones past its end that a short last item
    asks for)."""
    nx, ny, nz = shape
    kp, plane = dims(nx, ny, nz)
    nquads = nx * ny * (kp // V)
    q0 = np.arange(0, nquads + 2 * NT * 8, NT, dtype=np.int64)
    e0 = q0 * V
    e1 = e0 + NT * V
    for d in range(18):
        sh = shift(d, nx, ny, kp, eso, even)
        a = np.clip(e0 + sh - 1, 0, plane)
        z = np.clip(e1 + sh + 1, 0, plane)
        ok = a < z
        lo = (a[ok] * es) // 16 * 16
        hi = (z[ok] * es + 15) // 16 * 16
        assert (hi > lo).all() and (lo >= 0).all() and (hi <= plane * es).all(), d
    # Nu (FP32) spans
    a = np.clip(e0, 0, plane)
    z = np.clip(e1, 0, plane)
    ok = a < z
    assert ((z[ok] * 4 + 15) // 16 * 16 <= plane * 4).all()
