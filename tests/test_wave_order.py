"""The ticket order of the level-1 split's single-launch wavefront
(k_mis19_wave, hmfem_b200/csrc/rap_stencil.cu), restated on the CPU.

A warp holding ticket t resolves the x-row (j, k) that rows_before maps t
to, after the six rows that hold its cells' lower neighbours: (j, k-2),
(j-1, k-1), (j, k-1), (j+1, k-1), (j-2, k), (j-1, k).  Every wait ends only
if each of those rows has an earlier ticket (its warp took its ticket
before, so it is running or done) and the mapping covers every row once.
This checks both on every plane up to 14 x 14 and on the edges of large
ones, with the same integer formula as the kernel.
"""
import pytest

DEPS = [(0, -2), (-1, -1), (0, -1), (1, -1), (-2, 0), (-1, 0)]


def rows_before(t, ny, nz):
    """x-rows (j, k) of an ny x nz plane with j + 2k < t (the kernel's
    closed form)."""
    if t <= 0:
        return 0
    kf = (t - ny) // 2 + 1 if t >= ny else 0
    kp = (t + 1) // 2
    kf, kp = min(kf, nz), min(kp, nz)
    return ny * kf + (kp - kf) * t - (kp - kf) * (kf + kp - 1)


def row_of(tk, ny, nz):
    """The kernel's ticket -> (j, k): binary search for t, then k from the
    first row of that diagonal."""
    lo, hi = 0, (ny - 1) + 2 * (nz - 1)
    while lo < hi:
        mid = (lo + hi + 1) >> 1
        if rows_before(mid, ny, nz) <= tk:
            lo = mid
        else:
            hi = mid - 1
    t = lo
    kmin = (t - ny + 2) // 2 if t > ny - 1 else 0
    k = kmin + tk - rows_before(t, ny, nz)
    return t - 2 * k, k


@pytest.mark.parametrize("ny", range(1, 15))
def test_every_row_once_and_its_rows_below_earlier(ny):
    for nz in range(1, 15):
        order = [row_of(tk, ny, nz) for tk in range(ny * nz)]
        assert sorted(order) == sorted((j, k) for j in range(ny) for k in range(nz))
        pos = {r: i for i, r in enumerate(order)}
        for (j, k), i in pos.items():
            for dj, dk in DEPS:
                d = (j + dj, k + dk)
                if d in pos:
                    assert pos[d] < i, (ny, nz, (j, k), d)


@pytest.mark.parametrize("ny,nz", [(256, 256), (4, 100000), (3000, 5), (1024, 1024)])
def test_closed_form_counts_on_large_planes(ny, nz):
    tmax = (ny - 1) + 2 * (nz - 1)
    assert rows_before(tmax + 1, ny, nz) == ny * nz
    for t in (1, 2, ny - 1, ny, ny + 1, tmax // 2, tmax):
        kmin = (t - ny + 2) // 2 if t > ny - 1 else 0
        kmax = min(t // 2, nz - 1)
        assert rows_before(t + 1, ny, nz) - rows_before(t, ny, nz) == max(0, kmax - kmin + 1)
    for tk in (0, 1, ny * nz // 3, ny * nz - 1):
        j, k = row_of(tk, ny, nz)
        assert 0 <= j < ny and 0 <= k < nz
