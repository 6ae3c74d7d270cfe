"""The forward convolution's tiling, checked on the CPU: `hmfem_conv3d_plan`
returns the plan `hmfem_conv3d_fwd` launches, and a numpy emulation of the
kernel's addressing -- halo tile per 16-channel chunk, MMA runs of 128
consecutive halo positions shifted per tap (or, with grouped x taps, per
(dy, dz) pair with the three dx products combined one row apart, boundary
rows exchanged between consecutive runs of a z plane and zero otherwise),
the epilogue's validity test -- must reproduce a direct 3x3x3 convolution,
write every output cell exactly once, keep every operand row inside its
stage (rows past the halo are NaN here, so a valid output that read one
would show it), and fit the tensor memory, the shared memory and the
descriptors' 14-bit fields."""
import numpy as np
import pytest

from hmfem_b200 import guess

SMEM_MAX = 232448  # B200 opt-in shared memory per block
NSM = 148


def _check_limits(p, cin, cout):
    assert p["ns"] >= 1 and p["nb"] in (1, 2)
    nacc = (3 if p["xg"] else 1) * cout
    assert p["nb"] * p["runs"] * nacc <= p["tmem_cols"] <= 512
    if p["xg"]:
        assert 3 * cout <= 256 and p["ntx"] == 1          # the tile spans the x extent
    assert p["hcp"] % 8 == 0 and p["hcp"] >= p["hc"] + 128
    assert p["stage_bytes"] == 32 * p["hcp"] + (0 if p["wres"] else 27 * cout * 32)
    wall = 27 * cout * cin * 2                      # all chunks' weights
    assert p["wres"] == (wall <= 64 * 1024)
    assert p["wbytes"] == (wall if p["wres"] else 0)
    assert 8 * (2 * p["ns"] + 2 * p["nb"] + 1) + 8 <= 128    # barriers, slot, flag
    used = p["wbytes"] + p["ns"] * p["stage_bytes"] + 128 + (108 * cout if p["xg"] else 0) + 4 * cout
    assert used <= p["smem_bytes"] <= SMEM_MAX
    assert p["smem_bytes"] > SMEM_MAX // 2          # one CTA per SM
    assert p["smem_bytes"] < (1 << 18)              # 14-bit descriptor addresses
    assert p["hcp"] < (1 << 14)                     # LBO = 16 * hcp bytes
    if p["row_mode"]:
        assert p["bx"] == 128 and p["rp"] == p["by"]
    else:
        assert p["ntx"] == 1   # plane mode spans the x extent
        assert p["rp"] == -(-(p["W"] * (p["by"] - 1) + p["bx"]) // 128)
    assert p["runs"] == p["bz"] * p["rp"]


def _run_starts(p):
    W, H = p["W"], p["H"]
    out = []
    for r in range(p["runs"]):
        if p["row_mode"]:
            plane, row = divmod(r, p["by"])
            out.append((1 + W * (row + 1) + W * H * (plane + 1), plane, row))
        else:
            plane, j = divmod(r, p["rp"])
            out.append((1 + W + W * H * (plane + 1) + 128 * j, plane, -1))
    return out


def emulate(x, w, dims, p):
    """out (n, cout) from x (n, cin) and w (27, cout, cin) the kernel's way."""
    nx, ny, nz = dims
    cin, cout = x.shape[1], w.shape[1]
    W, H, bx, by, bz = p["W"], p["H"], p["bx"], p["by"], p["bz"]
    grid = x.reshape(nz, ny, nx, cin)
    out = np.full((nz, ny, nx, cout), np.nan)
    written = np.zeros((nz, ny, nx), np.int32)
    q = np.arange(128)
    offs = [(t % 3 - 1) + W * ((t // 3) % 3 - 1) + W * H * (t // 9 - 1) for t in range(27)]
    for tz in range(p["ntz"]):
        for ty in range(p["nty"]):
            for tx in range(p["ntx"]):
                x0, y0, z0 = tx * bx - 1, ty * by - 1, tz * bz - 1
                halo = np.full((p["hcp"], cin), np.nan)   # past hc: never a valid input
                hq = np.arange(p["hc"])
                zi, rem = divmod(hq, W * H)
                yi, xi = divmod(rem, W)
                gx, gy, gz = x0 + xi, y0 + yi, z0 + zi
                g = (gx >= 0) & (gx < nx) & (gy >= 0) & (gy < ny) & (gz >= 0) & (gz < nz)
                halo[:p["hc"]] = 0.0
                halo[hq[g]] = grid[gz[g], gy[g], gx[g]]
                starts = _run_starts(p)
                if p["xg"]:
                    D = []
                    for q0, _, _ in starts:
                        d = np.zeros((128, 3, cout))
                        for g in range(9):
                            lo = q0 + W * (g % 3 - 1) + W * H * (g // 3 - 1)
                            assert 0 <= lo and lo + 128 <= p["hcp"]
                            for dx in range(3):
                                d[:, dx] += halo[lo:lo + 128] @ w[3 * g + dx].T
                        D.append(d)
                for r, (q0, plane, row) in enumerate(starts):
                    if p["xg"]:
                        rp = p["rp"]
                        same_prev = not p["row_mode"] and r > 0 and r % rp != 0
                        same_next = not p["row_mode"] and r + 1 < p["runs"] and (r + 1) % rp != 0
                        prev = D[r - 1][127, 0] if same_prev else np.zeros(cout)
                        nxt = D[r + 1][0, 2] if same_next else np.zeros(cout)
                        acc = (np.vstack([prev[None], D[r][:127, 0]]) + D[r][:, 1]
                               + np.vstack([D[r][1:, 2], nxt[None]]))
                    else:
                        acc = np.zeros((128, cout))
                        for t in range(27):
                            lo = q0 + offs[t]
                            assert 0 <= lo and lo + 128 <= p["hcp"]
                            acc += halo[lo:lo + 128] @ w[t].T
                    pos = q0 + q
                    zi, rem = divmod(pos, W * H)
                    yi, xi = divmod(rem, W)
                    gx, gy, gz = x0 + xi, y0 + yi, z0 + zi
                    v = (zi == plane + 1) & (yi >= 1) & (yi <= by) & (xi >= 1) & (xi <= bx)
                    if row >= 0:
                        v &= yi == row + 1
                    v &= (gx < nx) & (gy < ny) & (gz < nz)
                    out[gz[v], gy[v], gx[v]] = acc[v]
                    written[gz[v], gy[v], gx[v]] += 1
    assert (written == 1).all()
    return out.reshape(-1, cout)


def direct(x, w, dims):
    nx, ny, nz = dims
    cin, cout = x.shape[1], w.shape[1]
    g = np.zeros((nz + 2, ny + 2, nx + 2, cin))
    g[1:-1, 1:-1, 1:-1] = x.reshape(nz, ny, nx, cin)
    out = np.zeros((nz, ny, nx, cout))
    for t in range(27):
        dx, dy, dz = t % 3 - 1, (t // 3) % 3 - 1, t // 9 - 1
        out += g[1 + dz:1 + dz + nz, 1 + dy:1 + dy + ny, 1 + dx:1 + dx + nx] @ w[t].T
    return out.reshape(-1, cout)


@pytest.mark.parametrize("dims,cin,cout", [
    ((9, 7, 5), 16, 16), ((20, 16, 12), 32, 64), ((11, 6, 7), 96, 32),
    ((20, 16, 12), 48, 16), ((8, 12, 8), 32, 96), ((130, 5, 3), 16, 16),
    ((128, 9, 4), 16, 32), ((257, 3, 2), 48, 16), ((64, 10, 3), 16, 32),
    ((128, 7, 3), 48, 16), ((40, 9, 5), 16, 48), ((33, 20, 6), 32, 64),
    ((256, 3, 2), 48, 16), ((200, 4, 3), 16, 16)])
def test_emulated_tiling_matches_direct_convolution(dims, cin, cout):
    p = guess.conv_plan(dims, cin, cout, NSM, SMEM_MAX)
    _check_limits(p, cin, cout)
    assert p["row_mode"] == 0 or dims[0] >= 128
    rng = np.random.default_rng(dims[0] + cin)
    n = dims[0] * dims[1] * dims[2]
    x = rng.standard_normal((n, cin))
    w = rng.standard_normal((27, cout, cin))
    np.testing.assert_allclose(emulate(x, w, dims, p), direct(x, w, dims), rtol=1e-12,
                               atol=1e-10)


@pytest.mark.parametrize("dims", [(128, 128, 128), (64, 64, 64), (32, 32, 32),
                                  (256, 256, 256), (16, 16, 16), (100, 37, 9), (1, 1, 1)])
@pytest.mark.parametrize("cin,cout", sorted(guess._SHAPES))
def test_plans_of_the_network_shapes_fit(dims, cin, cout):
    p = guess.conv_plan(dims, cin, cout, NSM, SMEM_MAX)
    _check_limits(p, cin, cout)
    nx, ny, nz = dims
    assert p["ntx"] * p["bx"] >= nx and p["nty"] * p["by"] >= ny and p["ntz"] * p["bz"] >= nz
    # every operand row of every run and tap inside the stage
    W, H = p["W"], p["H"]
    lo = min(q0 for q0, _, _ in _run_starts(p)) - (1 + W + W * H)
    hi = max(q0 for q0, _, _ in _run_starts(p)) + 127 + (1 + W + W * H)
    assert lo >= 0 and hi < p["hcp"]


def test_invalid_channel_counts_are_rejected():
    with pytest.raises(Exception):
        guess.conv_plan((8, 8, 8), 24, 16)
