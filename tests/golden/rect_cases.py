"""Seeded dreamrect (rectangular transducer SIR) cases shared by the golden
generator and the tests. Each case: observation points Ro (mm), element size
a x b (mm), surface discretisation dx, dy (mm), dt (us), nt samples, delay
(us), normal velocity v, sound speed cp (m/s)."""
import numpy as np


def _line(n, x0, x1, z):
    x = np.linspace(x0, x1, n)
    return np.asfortranarray(np.stack([x, np.zeros(n), np.full(n, z)], 1))


def _cloud(seed, n, xr, yr, zr):
    rng = np.random.default_rng(seed)
    return np.asfortranarray(np.stack([rng.uniform(*xr, n), rng.uniform(*yr, n), rng.uniform(*zr, n)], 1))


RECT_CASES = {
    # the reference TFM test's element and field line (python/tests/test_das_tfm.py:25-96)
    "tfm_test_line": dict(Ro=_line(31, -25.0, 25.0, 10.0), a=0.4, b=50.0, dx=0.05, dy=0.05, dt=0.02, nt=2000,
                          delay=0.0, v=1.0, cp=1500.0),
    # square element, 3-D points around it, a delay
    "square_cloud": dict(Ro=_cloud(1, 24, (-4, 4), (-4, 4), (0.5, 12)), a=2.0, b=2.0, dx=0.05, dy=0.05,
                         dt=0.025, nt=600, delay=0.3, v=1.0, cp=1480.0),
    # points close to the surface (short distances, large amplitudes)
    "near_surface": dict(Ro=_cloud(2, 16, (-1.5, 1.5), (-1.5, 1.5), (0.05, 0.6)), a=3.0, b=1.0, dx=0.02, dy=0.02,
                         dt=0.01, nt=400, delay=0.0, v=1.0, cp=1500.0),
    # a short response window: samples fall before and after it (out of bounds)
    "window_oob": dict(Ro=_cloud(3, 20, (-10, 10), (-5, 5), (2, 30)), a=4.0, b=6.0, dx=0.1, dy=0.1, dt=0.05,
                       nt=180, delay=2.5, v=2.0, cp=1500.0),
    # negative delay, odd discretisation
    "neg_delay": dict(Ro=_cloud(4, 12, (-3, 3), (-3, 3), (5, 15)), a=1.3, b=0.7, dx=0.013, dy=0.021, dt=0.02,
                      nt=900, delay=-0.4, v=1.0, cp=1540.0),
}


def random_rect_case(seed):
    """A seeded random element, discretisation, sampling and 20 points, with one
    delay or one per point: returns (case, delay)."""
    rng = np.random.default_rng(100 + seed)
    a, b = rng.uniform(0.05, 12.0, 2)
    c = dict(Ro=np.asfortranarray(np.stack([rng.uniform(-15, 15, 20), rng.uniform(-15, 15, 20),
                                            rng.uniform(0.1, 40, 20)], 1)),
             a=a, b=b, dx=a / rng.integers(1, 120), dy=b / rng.integers(1, 120), dt=float(rng.choice([0.01, 0.05, 0.25])),
             nt=int(rng.integers(1, 3000)), v=float(rng.uniform(0.5, 2)), cp=float(rng.uniform(1000, 6000)))
    d = np.full((1, 1), rng.uniform(-3, 10)) if rng.random() < 0.6 else rng.uniform(-3, 10, (20, 1))
    return c, d
