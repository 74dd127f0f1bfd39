"""Parameters of the reference fixtures in tests/golden/ (made by
make_ref_fixtures.py from the reference's own gsi on a 16x12x8 grid)."""
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
SHAPE = (16, 12, 8)


def load(name):
    return np.load(os.path.join(GOLDEN, f"ref_{name}.npz"))


def info_rows(log: str):
    return [list(map(float, l.split()[2:])) for l in log.splitlines() if l.startswith("Step ")]


def mart_params(gb):
    p = gb.default_params(gb.GS_MODEL_MART, gb.GS_MODE_REFCOMPAT)
    p.nvariants = 4
    p.nx, p.ny, p.nz = SHAPE
    p.dx = p.dy = p.dz = 0.2
    p.dt = 0.01
    p.transition_temperature = 450
    p.weight_dislocation = 0.1
    p.noise_amp = 0.0
    t = 0.0063  # varianttensor of scripts/in.mart
    p.set_eigenstrain(np.array([[[0, t, t], [t, 0, t], [t, t, 0]], [[0, t, -t], [t, 0, -t], [-t, -t, 0]],
                                [[0, -t, t], [-t, 0, -t], [t, -t, 0]], [[0, -t, -t], [-t, 0, t], [-t, t, 0]]]))
    return p


def ramp_temperature(i: int, total: int, t0: float = 460.0, t1: float = 300.0) -> float:
    """GS::Run calls Fix(i/total); Dynamics_mart::Fix stores st + progress (et - st)
    as a string with six significant digits, and Calculate parses it back
    (src/gs.cu:204, src/dynamics_mart.cu:421-441) -- all in float."""
    f = np.float32
    prog = f(f(i) / f(total))
    T = f(f(t0) + prog * (f(t1) - f(t0)))
    return float(f(float("%g" % T)))


def precip_params(gb):
    p = gb.default_params(gb.GS_MODEL_PRECIPITATE, gb.GS_MODE_REFCOMPAT)
    p.nvariants = 4
    p.nx, p.ny, p.nz = SHAPE
    p.dx = p.dy = p.dz = 0.2
    p.noise_amp = 0.0
    a, b = 0.01126, 0.00709  # varianttensor of scripts/in.precipitate
    p.set_eigenstrain(np.array([[[-a, -b, -b], [-b, -a, -b], [-b, -b, -a]], [[-a, b, b], [b, -a, -b], [b, -b, -a]],
                                [[-a, b, -b], [b, -a, b], [-b, b, -a]], [[-a, -b, b], [-b, -a, b], [b, b, -a]]]))
    return p


def stress_params(gb, log: str):
    """The stress tensor is the one the reference's script engine evaluated
    (six significant digits), read back from its `writehere` output."""
    i = log.find("3 4 3 3 \n")
    vals = [float(x) for x in log[i + 9:].split(">>>")[0].split()]
    p = gb.default_params(gb.GS_MODEL_STRESS, gb.GS_MODE_REFCOMPAT)
    p.nvariants = 4
    p.nx, p.ny, p.nz = SHAPE
    p.dx = p.dy = p.dz = 0.2
    p.set_eigenstrain(np.array(vals[:36]).reshape(4, 3, 3))
    return p
