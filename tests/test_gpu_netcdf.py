"""GPU: grid files written straight from device grids (ocu_nc_writer_add_grid) read back equal
to the grids' interiors, in both precisions, for a cell-centred and a face-staggered grid."""
import numpy as np
import pytest

import opencurrent_b200 as ocu
from oracle import oracle_ctypes as O
from tests.test_gpu_parity import dev_grid

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dt", [ocu.F32, ocu.F64])
def test_device_grids_round_trip(dt, tmp_path):
    nx, ny, nz = 12, 10, 8
    npd = np.float64 if dt == ocu.F64 else np.float32
    rng = np.random.default_rng(4)
    Lp, Lu = O.layout(nx, ny, nz), O.layout(nx + 1, ny, nz)
    hp = rng.standard_normal(int(Lp.allocated)).astype(npd)
    hu = rng.standard_normal(int(Lu.allocated)).astype(npd)
    gp, gu = dev_grid(hp, dt, Lp), dev_grid(hu, dt, Lu)
    t = ocu.NC_DOUBLE if dt == ocu.F64 else ocu.NC_FLOAT
    path = str(tmp_path / "dev.nc")
    w = ocu.NetCDFGrid3DWriter()
    w.open(path, nx, ny, nz, 1 / nx, 1 / ny, 1 / nz)
    w.define_variable("p", t, ocu.GS_CENTER_POINT)
    w.define_variable("u", t, ocu.GS_U_FACE)
    w.add_data("p", gp, 0)
    w.add_data("u", gu, 0)
    w.close()
    r = ocu.NetCDFGrid3DReader()
    r.open(path)
    np.testing.assert_array_equal(r.read_variable("p"), O.interior(hp, Lp))
    np.testing.assert_array_equal(r.read_variable("u"), O.interior(hu, Lu))
    r.close()
