"""The limiter's sweep stop keeps every bit (CPU).

SLOPELIMITER5 (slopelimiter.F:3555-3637) clamps an element's three vertex
values to its nodes' bounds and then runs three redistribution sweeps that
restore the element mean.  `limit_wetdry` stops the sweeps as soon as one
would start from sumdif == +0 with every vx - vmin free of a sign bit: each
of that sweep's reductions is then +0, so it and every later sweep leave
every vertex value's bits as they are.  This test runs the sweeps as the
kernel writes them (IEEE double, round to nearest, no contraction; x / 3 is
the correctly rounded quotient, which the kernel's div3 reproduces bit for
bit) with and without the stop on a million elements drawn to hit ties,
signed zeros, means on their bounds and clamped vertices (and, built by
hand, -0 vertex values around a +0 mean, the case of the stop's sign
guard), and compares the vertex values bit for bit.  The device build is
checked against the oracle on real decks by the strict GPU tests; this pins
the stop's argument on inputs no deck reaches.
"""
import numpy as np

# p=1 basis at the corners (modes 2 and 3), as the kernel's phi_corner
PHI = np.array([[-1.0, -1.0], [-1.0, 1.0], [2.0, 0.0]])


def div_count(x, kdp):
    """x / max(1, kdp) for kdp in {0, 1, 2, 3}, as the kernel forms it."""
    return np.where(kdp <= 1, x, np.where(kdp == 2, x * 0.5, x / 3.0))


def sweeps(vx, vmin, vmax, z0, stop):
    vx = vx.copy()
    done = np.zeros(len(z0), bool)
    stopped = np.zeros(len(z0), int)
    for sweep in range(3):
        sumloc = (vx[:, 0] + vx[:, 1] + vx[:, 2]) / 3.0
        sumdif = (sumloc - z0) * 3.0
        if stop:
            quiet = (sumdif == 0.0) & ~np.signbit(sumdif) & ~np.signbit(vx - vmin).any(axis=1)
            stopped += quiet & ~done
            done |= quiet
        signdif = np.copysign(1.0, sumdif)
        dif = (vx - z0[:, None]) * signdif[:, None]
        kdp = (dif > 0).sum(axis=1)
        for k in range(3):
            pos = dif[:, k] > 0
            redfac = np.where(pos, div_count(sumdif * signdif, kdp), 0.0)
            kdp = np.where(pos, kdp - 1, kdp)
            redmax = np.where(signdif > 0, vx[:, k] - vmin[:, k], vmax[:, k] - vx[:, k])
            redfac = np.fmin(redfac, redmax)
            sumdif = sumdif - redfac * signdif
            vx[:, k] = np.where(done, vx[:, k], vx[:, k] - redfac * signdif)
    return vx, stopped


def elements(rng, n):
    """Element means, modes 2-3 and node bounds that contain the mean,
    mixing smooth values, exact ties (small dyadic numbers), zeros of both
    signs and bounds equal to the mean."""
    kind = rng.integers(0, 4, n)
    z0 = np.where(kind == 0, rng.normal(0.0, 1.0, n),
                  np.where(kind == 1, rng.integers(-8, 9, n) / 8.0,
                           np.where(kind == 2, 0.0, 20.0 + rng.normal(0.0, 1e-3, n))))
    z0 = np.where(rng.random(n) < 0.05, -0.0, z0)
    scale = np.where(kind == 1, 1 / 16.0, 10.0 ** rng.uniform(-9, 0, n))
    z1 = np.where(rng.random(n) < 0.1, 0.0, rng.normal(0.0, 1.0, n) * scale)
    z2 = np.where(rng.random(n) < 0.1, -0.0, rng.normal(0.0, 1.0, n) * scale)
    z1 = np.where(kind == 1, np.round(z1 * 64) / 64, z1)
    lo = np.abs(rng.normal(0.0, 1.0, (n, 3))) * scale[:, None] * rng.choice([0.0, 0.5, 2.0], (n, 3))
    hi = np.abs(rng.normal(0.0, 1.0, (n, 3))) * scale[:, None] * rng.choice([0.0, 0.5, 2.0], (n, 3))
    vmin, vmax = z0[:, None] - lo, z0[:, None] + hi
    vx = (z0[:, None] + PHI[None, :, 0] * z1[:, None]) + PHI[None, :, 1] * z2[:, None]
    vx = np.fmax(np.fmin(vx, vmax), vmin)
    return vx, vmin, vmax, z0


def signed_zero_elements():
    """Vertex values -0 around a mean +0: sumdif = (-0 - 0) * 3 = -0, the
    sweep's signdif is -1 and vx - (+0)(-1) turns each -0 into +0.  A stop
    at sumdif == -0 would keep the -0 bits."""
    vx = np.full((4, 3), -0.0)
    vx[1, 2] = 0.0
    vmin = np.array([[-1.0] * 3, [-0.5] * 3, [-0.0] * 3, [-2.0, -0.0, -1.0]])
    vmax = np.array([[1.0] * 3, [0.5] * 3, [0.0] * 3, [2.0, 0.0, 1.0]])
    return vx, vmin, vmax, np.zeros(4)


def test_sweep_stop_is_bit_exact():
    rng = np.random.default_rng(20261204)
    total_stopped = 0
    for block in range(5):
        vx, vmin, vmax, z0 = elements(rng, 250_000) if block < 4 else signed_zero_elements()
        full, _ = sweeps(vx, vmin, vmax, z0, stop=False)
        short, stopped = sweeps(vx, vmin, vmax, z0, stop=True)
        np.testing.assert_array_equal(full.view(np.int64), short.view(np.int64))
        total_stopped += int(stopped.sum())
    # the stop is taken on most elements, so the comparison exercises it
    assert total_stopped > 500_000
