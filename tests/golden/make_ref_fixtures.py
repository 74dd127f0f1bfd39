"""Generate golden fixtures by running the reference's own gsi
(oracle/_ref/gsi, built by oracle/build_ref.sh from the reference sources)
on small seeded inputs.  The physics cases need a CUDA device (the
reference's kernels are device-only); the front-end cases run anywhere.

  REF=<reference tree> python tests/golden/make_ref_fixtures.py --out DIR [--physics] [--frontend]

REF (required for --frontend) names the reference tree whose scripts/ the
front-end cases read.

Writes DIR/ref_<case>.npz (inputs, dumps, the info lines),
DIR/frontend_<script>.txt and DIR/ref_cores.npz (the nuclei generator, which
runs on the host in the reference).  The committed copies under tests/golden/ are
the outputs of this script; the tests never run the reference.
"""
from __future__ import annotations

import argparse
import os
import shutil
import struct
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
GSI = os.path.join(ROOT, "oracle", "_ref", "gsi")

MART_TENSOR = """3 4 3 3
0.00 0.0063 0.0063  0.0063 0.0 0.0063    0.0063 0.0063 0.0
0.00 0.0063 -0.0063  0.0063 0.0 -0.0063 -0.0063 -0.0063 0.0
0.00 -0.0063 0.0063  -0.0063 0.0 -0.0063  0.0063 -0.0063 0.0
0.00 -0.0063 -0.0063  -0.0063 0.0 0.0063  -0.0063 0.0063 0.0"""

PRECIP_TENSOR = """3 4 3 3
-0.01126 -0.00709 -0.00709 -0.00709 -0.01126 -0.00709 -0.00709 -0.00709 -0.01126
-0.01126 0.00709 0.00709 0.00709 -0.01126 -0.00709 0.00709 -0.00709 -0.01126
-0.01126 0.00709 -0.00709 0.00709 -0.01126 0.00709 -0.00709 0.00709 -0.01126
-0.01126 -0.00709 0.00709 -0.00709 -0.01126 0.00709 0.00709 0.00709 -0.01126"""

# the expression block of the stress script (values evaluated by the script engine)
STRESS_TENSOR = """3 4 3 3
{
-1.835*0.01, -8.1868274*0.001, -5.7889605*0.001,-8.1868256*0.001, -8.897*0.001, -3.3422573*0.001,-5.7889605*0.001, -3.3422580*0.001, -6.54*0.001
-4.17*0.001,  0.0,  0.0, 0.0, -2.3*0.01, 6.6845156*0.001, 0.0,  6.6845166*0.001, -6.5*0.001
-4.17*0.001,  0.0,  0.0, 0.0, -4.17*0.001, 0.0,0.0,  0.0, -2.544*0.01
-1.835*0.01,  8.1868265*0.001,  5.788961*0.001,8.1868256*0.001, -8.897*0.001, -3.3422573*0.001,5.7889605*0.001, -3.3422580*0.001, -6.5*0.001
}"""

SHAPE = (16, 12, 8)


def write_text_field(path: str, arr: np.ndarray) -> None:
    """The reference's text field format: 'ndim d1 .. dn' then one value per line."""
    a = np.asarray(arr, dtype=np.float32)
    with open(path, "w") as f:
        f.write(" ".join(str(x) for x in [a.ndim, *a.shape]) + " \n")
        f.write("\n".join(repr(float(x)) for x in a.ravel()) + "\n")


def read_binary_field(path: str) -> np.ndarray:
    """The reference's binary field format: int32 ndim, int32 dims, float32 values."""
    with open(path, "rb") as f:
        nd = struct.unpack("i", f.read(4))[0]
        dims = struct.unpack("i" * nd, f.read(4 * nd))
        vals = np.frombuffer(f.read(), dtype=np.float32)
    return vals.reshape(dims)


def mart_inputs():
    rng = np.random.default_rng(7)
    nx, ny, nz = SHAPE
    eta = rng.uniform(0.0, 0.1, (4, nx, ny, nz)).astype(np.float32)
    ds = rng.uniform(-0.05, 0.05, (6, nx, ny, nz)).astype(np.float32)
    defect = (rng.random((nx, ny, nz)) < 0.05).astype(np.float32)
    return {"data.eta": eta, "data.stress": ds, "data.defect": defect}


def mart_script() -> str:
    nx, ny, nz = SHAPE
    return f"""sys mart
set binary off
set gridsize {nx} {ny} {nz} 0.2 0.2 0.2
set deltatime 0.01
set transitiontemperature 450
set weightdislocation .1
set weightnoise 0
read eta data.eta
read dislocationstress data.stress
read defect data.defect
readhere varianttensor
{MART_TENSOR}
info 5 temperature eta gradient chemical elastic dislocation
set binary on
dump dumpdir 5 eta
set fix temperature 460 300
run 5
"""


def precip_inputs():
    rng = np.random.default_rng(8)
    nx, ny, nz = SHAPE
    eta = rng.uniform(0.0, 0.5, (4, nx, ny, nz)).astype(np.float32)
    con = (0.2 + rng.uniform(-0.02, 0.02, (nx, ny, nz))).astype(np.float32)
    return {"data.eta": eta, "data.con": con}


def precip_script() -> str:
    nx, ny, nz = SHAPE
    return f"""sys precipitate
set binary off
set gridsize {nx} {ny} {nz} 0.2 0.2 0.2
set deltatime 0.1
set coefficient 54.00 -17.0 7.0 2.5 0.2 0.2 0.2
set arfi 300.0
set beta 300.0
set meta 0.4
set lpp  0.4
set xi   400
set concentration 0.1 0.44
set weightnoise 0
read eta data.eta
read concentration data.con
readhere varianttensor
{PRECIP_TENSOR}
info 5 eta_average
set binary on
dump dumpdir 5 eta concentration
run 5
"""


def stress_inputs():
    rng = np.random.default_rng(9)
    nx, ny, nz = SHAPE
    return {"data.eta": rng.uniform(0.0, 1.0, (4, nx, ny, nz)).astype(np.float32)}


def stress_script() -> str:
    nx, ny, nz = SHAPE
    return f"""sys stress
set binary off
set gridsize {nx} {ny} {nz} 0.2 0.2 0.2
read eta data.eta
readhere varianttensor
{STRESS_TENSOR}
writehere varianttensor
set binary on
dump dumpdir 1 stress defect
run 1
"""


def run_case(gsi: str, workdir: str, inputs: dict, script: str, name: str) -> str:
    """Write the inputs (text format) and the script, run a gsi binary."""
    for fn, arr in inputs.items():
        write_text_field(os.path.join(workdir, fn), arr)
    path = os.path.join(workdir, name)
    with open(path, "w") as f:
        f.write(script)
    r = subprocess.run([gsi, name], cwd=workdir, capture_output=True, text=True, timeout=600)
    return r.stdout


def case_mart(out: str) -> None:
    inputs = mart_inputs()
    with tempfile.TemporaryDirectory() as d:
        log = run_case(GSI, d, inputs, mart_script(), "in.mart16")
        dumps = np.stack([read_binary_field(os.path.join(d, "dumpdir", f"eta.{i}.data")) for i in range(1, 6)])
    np.savez_compressed(os.path.join(out, "ref_mart.npz"), eta0=inputs["data.eta"],
                        dislocationstress=inputs["data.stress"], defect=inputs["data.defect"],
                        eta_steps=dumps, log=np.array(log))


def case_precipitate(out: str) -> None:
    inputs = precip_inputs()
    with tempfile.TemporaryDirectory() as d:
        log = run_case(GSI, d, inputs, precip_script(), "in.precipitate16")
        e = np.stack([read_binary_field(os.path.join(d, "dumpdir", f"eta.{i}.data")) for i in range(1, 6)])
        c = np.stack([read_binary_field(os.path.join(d, "dumpdir", f"concentration.{i}.data")) for i in range(1, 6)])
    np.savez_compressed(os.path.join(out, "ref_precipitate.npz"), eta0=inputs["data.eta"], con0=inputs["data.con"],
                        eta_steps=e, con_steps=c, log=np.array(log))


def case_stress(out: str) -> None:
    inputs = stress_inputs()
    with tempfile.TemporaryDirectory() as d:
        log = run_case(GSI, d, inputs, stress_script(), "in.stress16")
        stress = read_binary_field(os.path.join(d, "dumpdir", "stress.1.data"))
        defect = read_binary_field(os.path.join(d, "dumpdir", "defect.1.data"))
    np.savez_compressed(os.path.join(out, "ref_stress.npz"), eta0=inputs["data.eta"], stress=stress, defect=defect,
                        log=np.array(log))


def case_frontend(out: str) -> None:
    for name in ["in.if.loop.while", "in.pow", "in.expr"]:
        src = os.path.join(os.environ["REF"], "scripts", name)
        if not os.path.exists(src):
            src = os.path.join(HERE, "scripts", name)  # project scripts in the reference's language
        with tempfile.TemporaryDirectory() as d:
            shutil.copy(src, os.path.join(d, name))
            r = subprocess.run([GSI, name], cwd=d, capture_output=True, text=True, timeout=60)
        with open(os.path.join(out, f"frontend_{name.replace('.', '_')}.txt"), "w") as f:
            f.write(r.stdout)


CORES_CASES = [  # (name, grid, variants, nuclei, radius, method)
    ("random", (32, 24, 16), 4, 3, 4.5, "random"),
    ("random_dense", (16, 16, 16), 3, 8, 5.0, "random"),
    ("regular", (24, 20, 32), 4, 2, 3.0, "regular"),
]


def cores_script(grid, V, n, r, method) -> str:
    nx, ny, nz = grid
    return f"""sys cores
set gridsize {nx} {ny} {nz} 0.2 0.2 0.2
set variantn {V}
set coresn {n}
set radius {r}
set concentration 0.2 0.44
set method {method}
set binary on
dump dd 1 eta concentration
run
"""


def case_cores(out: str) -> None:
    """Dynamics_cores runs on the host in the reference: no device needed."""
    arrays = {}
    for name, grid, V, n, r, method in CORES_CASES:
        with tempfile.TemporaryDirectory() as d:
            with open(os.path.join(d, "in.cores"), "w") as f:
                f.write(cores_script(grid, V, n, r, method))
            subprocess.run([GSI, "in.cores"], cwd=d, capture_output=True, text=True, timeout=120)
            arrays[f"{name}_eta"] = read_binary_field(os.path.join(d, "dd", "eta.1.data"))
            arrays[f"{name}_concentration"] = read_binary_field(os.path.join(d, "dd", "concentration.1.data"))
    np.savez_compressed(os.path.join(out, "ref_cores.npz"), **arrays)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--physics", action="store_true")
    ap.add_argument("--frontend", action="store_true")
    a = ap.parse_args()
    os.makedirs(a.out, exist_ok=True)
    if a.frontend:
        case_frontend(a.out)
        case_cores(a.out)
    if a.physics:
        case_mart(a.out)
        case_precipitate(a.out)
        case_stress(a.out)


if __name__ == "__main__":
    main()
