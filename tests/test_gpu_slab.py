"""The slab-decomposed martensite step (gs_slab_*) on one GPU: R slabs in one
process, the all-to-all transposes and the halo exchange done as device
copies (no kernel waits on another).  Every line transform, table point and
cell update is the one-device step's own arithmetic, so the slabs must give
the one-device fields bit for bit; FP64 is also held to the FP64 oracle
(1e-11 relative L2, the tolerance of the one-device parity tests)."""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu
F64, F32 = 1, 0


def params(gb, shape, dtype, V=3, noise=1e-3):
    p = gb.mart3d_params(16, dtype=dtype, noise=noise)
    p.nx, p.ny, p.nz = shape
    if V != 3:
        p.nvariants = V
        p.set_eigenstrain(gb.tetragonal_eigenstrains(V, 0.02, -0.01))
    return p


def one_device(gb, p, eta0, steps):
    s = gb.Sim(p)
    try:
        s.set_field("eta", eta0)
        s.step(steps)
        return s.eta(np.float64)
    finally:
        s.close()


@pytest.mark.parametrize("shape,V,R,dtype", [
    ((16, 12, 32), 3, 2, F32),
    ((16, 12, 32), 3, 4, F64),
    ((8, 8, 16), 2, 8, F32),      # one x-plane per slab: both halos from neighbours
    ((32, 16, 64), 4, 4, F32),
    ((64, 64, 64), 3, 2, F32),
    ((12, 8, 24), 3, 2, F64),     # radix-3 lengths
])
def test_slabs_equal_one_device_bit_for_bit(gb, shape, V, R, dtype):
    import gs_slab

    p = params(gb, shape, dtype, V)
    eta0 = gb.initial_eta(p, 7, 0.4)
    if dtype == F32:
        eta0 = eta0.astype(np.float32).astype(np.float64)
    ref = one_device(gb, p, eta0, 3)
    got = gs_slab.run_local(p, eta0, 3, R)
    assert np.isfinite(got).all()
    assert np.array_equal(got, ref)


def test_slabs_fp64_match_oracle(gb, orc):
    import gs_slab

    p = params(gb, (16, 8, 24), F64)
    eta0 = gb.initial_eta(p, 8, 0.5)
    got = gs_slab.run_local(p, eta0, 2, 4)
    assert rel_l2(got, orc.mart_run(p, eta0, 2)) < 1e-11


def test_slab_geometry_and_rejections(gb):
    import gs_slab

    p = params(gb, (16, 12, 32), F32)
    s = gs_slab.Slab(p, 1, 4)
    try:
        g = s.geom
        assert (g.x0, g.nx_local, g.kz0, g.nkz_local) == (4, 4, 4, 4)
        assert g.a2a_bytes == 3 * 4 * 12 * 32 * 4
        assert g.halo_bytes == 2 * 3 * 12 * 32 * 4
    finally:
        s.close()
    with pytest.raises(RuntimeError):
        gs_slab.Slab(params(gb, (16, 12, 32), F32), 0, 3)  # 16 planes over 3 ranks
    with pytest.raises(RuntimeError):
        gs_slab.Slab(params(gb, (16, 12, 1), F32), 0, 2)   # a 2D grid is not split
    with pytest.raises(RuntimeError):
        gs_slab.Slab(params(gb, (16, 12, 32), F32), 4, 4)  # rank out of range
