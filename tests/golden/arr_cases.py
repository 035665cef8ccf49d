"""Seeded dream_arr_rect (array of rectangular elements) cases shared by the
golden generator and the tests. Each case: observation points Ro (mm),
element size a x b and discretisation dx, dy (mm), element centres G
(M x 3, mm), dt (us), nt, delay (us, scalar or per point), v, cp (m/s),
focusing / steering / apodisation settings and the error level."""
import numpy as np


def _cloud(seed, n, xr, yr, zr):
    rng = np.random.default_rng(seed)
    return np.asfortranarray(np.stack([rng.uniform(*xr, n), rng.uniform(*yr, n), rng.uniform(*zr, n)], 1))


def _grid(xs, ys, z=0.0):
    gx, gy = np.meshgrid(xs, ys)
    gx, gy = gx.reshape(-1, order="F"), gy.reshape(-1, order="F")
    return np.asfortranarray(np.stack([gx, gy, np.full(gx.size, z)], 1))


def _case(Ro, a, b, G, dx, dy, dt, nt, delay, v=1.0, cp=1500.0, foc_met="off", focal=0.0, steer_met="off",
          theta=0.0, phi=0.0, apod_met="off", apod=None, apod_par=0.0, err="ignore"):
    return dict(Ro=np.asfortranarray(Ro, dtype=np.float64), a=a, b=b, G=np.asfortranarray(G, dtype=np.float64),
                dx=dx, dy=dy, dt=dt, nt=nt, delay=delay, v=v, cp=cp, foc_met=foc_met, focal=focal,
                steer_met=steer_met, theta=theta, phi=phi, apod_met=apod_met, apod=apod, apod_par=apod_par, err=err)


_lin21 = np.stack([np.linspace(-10.0, 10.0, 21), np.zeros(21), np.zeros(21)], 1)
_rng = np.random.default_rng(11)

ARR_CASES = {
    # the reference's Python test (python/tests/test_dream_arr_rect.py): 21 elements of
    # 0.8 x 20 mm along x, focused at 10 mm, one point on axis
    "reference_test": _case(np.array([[0.0, 0.0, 10.0]]), 0.8, 20.0, _lin21, 0.05, 0.05, 0.25, 300, 0.0, 1.0,
                            1000.0, foc_met="x", focal=10.0),
    # the same array over a line of points at the focal depth and off it
    "reference_line": _case(np.stack([np.linspace(-12, 12, 25), np.zeros(25), np.linspace(4, 20, 25)], 1), 0.8, 20.0,
                            _lin21, 0.05, 0.05, 0.25, 300, 0.0, 1.0, 1000.0, foc_met="x", focal=10.0),
    # 2-D array of the reference's example (examples/rect_arr_example.m) on a 5 x 5 grid:
    # xy focusing at 50 mm, steering -25 degrees in x, a 2 mm time window at 49-51 mm
    "example_steered": _case(np.stack([np.linspace(-20, 20, 30), np.zeros(30), np.linspace(30, 70, 30)], 1),
                             0.9, 0.9, _grid(np.arange(-2.0, 3.0), np.arange(-2.0, 3.0)), 0.03, 0.03, 0.1, 13,
                             49.0 * 1e3 / 1500.0, foc_met="xy", focal=50.0, steer_met="x", theta=-25.0),
    # along y: y focusing, y steering, Hann apodisation, one delay per point
    "y_hann": _case(_cloud(5, 18, (-3, 3), (-6, 6), (4, 14)), 1.5, 0.6, np.stack([np.zeros(8), np.linspace(-3.5, 3.5, 8),
                    np.zeros(8)], 1), 0.05, 0.04, 0.02, 900, np.linspace(0.0, 1.0, 18), foc_met="y", focal=8.0,
                    steer_met="y", phi=10.0, apod_met="hann"),
    # x+y focusing, xy steering, clamped apodisation on a 3 x 4 grid
    "x_y_clamped": _case(_cloud(6, 14, (-5, 5), (-5, 5), (6, 16)), 1.0, 1.2, _grid(np.linspace(-2, 2, 3),
                         np.linspace(-3, 3, 4)), 0.05, 0.05, 0.025, 800, 0.2, foc_met="x+y", focal=11.0,
                         steer_met="xy", theta=7.5, phi=-12.0, apod_met="clamped"),
    # user-defined delays and weights, elements off the z = 0 plane, 'warn'
    "ud_3d": _case(_cloud(7, 16, (-4, 4), (-4, 4), (5, 12)), 0.7, 0.9, _cloud(8, 9, (-3, 3), (-3, 3), (-0.5, 0.5)),
                   0.05, 0.05, 0.02, 700, -0.3, foc_met="ud", focal=_rng.uniform(0.0, 0.8, 9), apod_met="ud",
                   apod=_rng.uniform(0.2, 1.5, 9), err="warn"),
    # triangle / gauss / raised / hamming / simply windows on one line array
    "triangle": _case(_cloud(9, 10, (-4, 4), (-1, 1), (3, 9)), 0.5, 3.0, np.stack([np.linspace(-3, 3, 7),
                      np.zeros(7), np.zeros(7)], 1), 0.05, 0.1, 0.02, 600, 0.0, apod_met="triangle"),
    "gauss_raised": _case(_cloud(10, 10, (-4, 4), (-1, 1), (3, 9)), 0.5, 3.0, np.stack([np.linspace(-3, 3, 7),
                          np.zeros(7), np.zeros(7)], 1), 0.05, 0.1, 0.02, 600, 0.0, apod_met="raised",
                          apod_par=0.0),
    "hamming_simply": _case(_cloud(12, 10, (-4, 4), (-1, 1), (3, 9)), 0.5, 3.0, np.stack([np.linspace(-3, 3, 7),
                            np.zeros(7), np.zeros(7)], 1), 0.05, 0.1, 0.02, 600, 0.0, apod_met="hamming"),
    # fewer than 32 surface terms per element (2 x 2): one warp step spans several elements
    "tiny_elements": _case(_cloud(13, 12, (-6, 6), (-6, 6), (2, 10)), 0.1, 0.1, _grid(np.linspace(-4, 4, 9),
                           np.linspace(-4, 4, 7)), 0.05, 0.05, 0.01, 1400, 0.0, foc_met="xy", focal=6.0,
                           apod_met="simply"),
    # a short window: most elements miss it entirely, some straddle its ends
    "dead_elements": _case(_cloud(14, 24, (-15, 15), (-2, 2), (10, 40)), 1.0, 1.0, _grid(np.linspace(-8, 8, 17),
                           np.array([0.0])), 0.05, 0.05, 0.05, 40, 18.0 * 1e3 / 1500.0, foc_met="x", focal=20.0,
                           steer_met="x", theta=15.0),
    # windows longer than shared memory holds: accumulated in the output columns
    "global_window": _case(_cloud(16, 8, (-20, 20), (-2, 2), (5, 20)), 0.5, 0.5, np.array([[-30.0, 0.0, 0.0],
                           [0.0, 0.0, 0.0], [30.0, 0.0, 0.0]]), 0.05, 0.05, 0.001, 30000, 0.0, foc_met="x",
                           focal=12.0),
    # one element at the origin: dreamrect
    "single_origin": _case(_cloud(15, 12, (-3, 3), (-3, 3), (1, 9)), 2.0, 1.5, np.zeros((1, 3)), 0.05, 0.05,
                           0.02, 700, 0.1),
    # sample magnitudes above the proven-window range (dt = 1 ps at 1 m): unbounded windows
    "fine_sampling": _case(np.stack([np.linspace(-0.05, 0.05, 6), np.zeros(6), np.full(6, 1000.0)], 1), 0.2, 0.2,
                           np.array([[0.0, 0.0, 0.0], [0.02, 0.01, 0.0]]), 0.01, 0.01, 1e-6, 6000,
                           1000.0 * 1e3 / 1500.0),
}

# method names accepted by dream_arr_rect (the keys of oracle.FOC_METHODS, ...)
FOC_NAMES = ["off", "x", "y", "xy", "on", "x+y", "ud"]
STEER_NAMES = ["off", "x", "y", "xy"]
APOD_NAMES = ["off", "triangle", "gauss", "raised", "hann", "hamming", "simply", "clamped", "ud"]


def random_case(seed):
    """A seeded random array, sampling and method choice (small enough for the oracle)."""
    rng = np.random.default_rng(seed)
    M = int(rng.integers(1, 40))
    a, b = rng.uniform(0.05, 2.0, 2)
    dx, dy = a / rng.integers(1, 40), b / rng.integers(1, 40)
    G = np.asfortranarray(np.stack([rng.uniform(-6, 6, M), rng.uniform(-6, 6, M), rng.uniform(-0.5, 0.5, M)], 1))
    No = int(rng.integers(1, 24))
    Ro = np.asfortranarray(np.stack([rng.uniform(-10, 10, No), rng.uniform(-10, 10, No), rng.uniform(0.2, 25, No)], 1))
    cp = float(rng.uniform(1000, 6000))
    dt = float(rng.choice([0.005, 0.02, 0.1, 0.25]))
    nt = int(rng.integers(1, 2500))
    delay = float(rng.uniform(-2, 8)) if rng.random() < 0.7 else rng.uniform(-2, 8, No)
    foc = str(rng.choice(list(FOC_NAMES)))
    steer = str(rng.choice(list(STEER_NAMES)))
    apod = str(rng.choice(list(APOD_NAMES)))
    return dict(Ro=Ro, a=a, b=b, G=G, dx=dx, dy=dy, dt=dt, nt=nt, delay=delay, v=float(rng.uniform(0.5, 2)), cp=cp,
                foc_met=foc, focal=rng.uniform(0, 1, M) if foc == "ud" else float(rng.uniform(2, 30)),
                steer_met=steer, theta=float(rng.uniform(-40, 40)), phi=float(rng.uniform(-40, 40)),
                apod_met=apod, apod=rng.uniform(0.1, 1.5, M) if apod == "ud" else None, apod_par=0.0, err="ignore")
