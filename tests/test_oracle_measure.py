"""The oracle's measurements -- axis_pair_sums (src/models/mod.rs:44-61),
Z2Gauge::polyakov_loop (gauge/mod.rs:179-212) and wilson_rectangles
(gauge/mod.rs:226-274) -- against an independent numpy restatement, the
reference's anchors (C_0 = 1, cold configuration = 1 everywhere) and gauge
invariance."""
import numpy as np
import pytest


def _grid(shape, a):
    # reference order: direction 0 fastest -> numpy axes reversed
    return a.reshape(tuple(reversed(shape)))


def _shift(g, d, mu, k):
    # value at x + k * e_mu
    return np.roll(g, -k, axis=d - 1 - mu)


def np_pair_sums(shape, cfg, ising):
    d = len(shape)
    g = _grid(shape, cfg.astype(np.int64))
    rows = []
    for mu in range(d):
        row = []
        for r in range(shape[mu] // 2 + 1):
            h = _shift(g, d, mu, r)
            row.append(int(((1 - 2 * g) * (1 - 2 * h)).sum()) if ising else int((g == h).sum()))
        rows.append(np.array(row))
    return rows


def _links(shape, cfg):
    d = len(shape)
    n = int(np.prod(shape))
    return [_grid(shape, cfg.reshape(n, d)[:, mu].astype(np.int64)) for mu in range(d)]


def _line(U, d, mu, x_shift_fn, r):
    acc = np.zeros_like(U[mu])
    for k in range(r):
        acc ^= _shift(U[mu], d, mu, k)
    return acc


def np_wilson(shape, cfg, max_side):
    d = len(shape)
    U = _links(shape, cfg)
    mx = min(max_side, min(shape) // 2)
    totals = np.zeros((mx + 1, mx + 1), dtype=np.int64)
    for r in range(1, mx + 1):
        for t in range(1, mx + 1):
            tot = 0
            for mu in range(d):
                for nu in range(d):
                    if mu == nu:
                        continue
                    lm = _line(U, d, mu, None, r)  # line_mu(x, r)
                    ln = _line(U, d, nu, None, t)  # line_nu(x, t)
                    w = lm ^ _shift(ln, d, mu, r) ^ _shift(lm, d, nu, t) ^ ln
                    tot += int((1 - 2 * w).sum())
            totals[r, t] = tot
    return totals, d * (d - 1) * int(np.prod(shape))


def np_polyakov(shape, cfg, direction):
    d = len(shape)
    U = _links(shape, cfg)
    line = _line(U, d, direction, None, shape[direction])
    lines = int(np.prod(shape)) // shape[direction]
    # every starting point of a line gives the same product: count one per line
    return int((1 - 2 * line).sum()) // shape[direction], lines


@pytest.mark.parametrize("shape", [(8,), (6, 4), (4, 6, 2), (4, 2, 4, 2)])
@pytest.mark.parametrize("kind,q", [("ising", 2), ("potts", 3), ("potts", 5)])
def test_axis_pair_sums(oracle, shape, kind, q):
    lat = oracle.Lattice(shape)
    model = oracle.Model.ising(1.0, 0.0) if kind == "ising" else oracle.Model.potts(q, 1.0)
    rng = np.random.default_rng(sum(shape) + q)
    n = int(np.prod(shape))
    for cfg in (np.zeros(n, np.uint8), rng.integers(0, q, n).astype(np.uint8)):
        got = oracle.axis_pair_sums(model, lat, cfg)
        want = np_pair_sums(shape, cfg, kind == "ising")
        assert [list(x) for x in got] == [list(x) for x in want]
        for row in got:
            assert row[0] == n  # the C_0 anchor: every site pairs with itself
        if not cfg.any():
            assert all((row == n).all() for row in got)


@pytest.mark.parametrize("shape", [(4, 4), (6, 4, 4), (4, 4, 4, 4), (6, 4, 2, 4)])
def test_wilson_and_polyakov(oracle, shape):
    d = len(shape)
    lat = oracle.Lattice(shape)
    n = int(np.prod(shape))
    rng = np.random.default_rng(d)
    cold = np.zeros(n * d, np.uint8)
    tot, pl = oracle.wilson_totals(lat, cold, 8)
    assert (tot[1:, 1:] == pl).all()  # cold: every loop is +1
    for direction in range(d):
        assert oracle.polyakov_sum(lat, cold, direction) == (n // shape[direction], n // shape[direction])
    cfg = rng.integers(0, 2, n * d).astype(np.uint8)
    tot, pl = oracle.wilson_totals(lat, cfg, 8)
    want, wpl = np_wilson(shape, cfg, 8)
    assert pl == wpl and (tot == want).all()
    assert (tot == tot.T).all()  # both orientations of every plane are averaged together
    for direction in range(d):
        assert oracle.polyakov_sum(lat, cfg, direction) == np_polyakov(shape, cfg, direction)
    # a gauge transformation (flip every link touching one site) changes no loop
    g = cfg.reshape(n, d).copy()
    site = 5 % n
    coords = np.unravel_index(site, tuple(reversed(shape)))[::-1]
    for mu in range(d):
        g[site, mu] ^= 1
        back = list(coords)
        back[mu] = (back[mu] - 1) % shape[mu]
        g[np.ravel_multi_index(tuple(reversed(back)), tuple(reversed(shape))), mu] ^= 1
    g = g.reshape(-1)
    assert (oracle.wilson_totals(lat, g, 8)[0] == tot).all()
    for direction in range(d):
        assert oracle.polyakov_sum(lat, g, direction) == oracle.polyakov_sum(lat, cfg, direction)
