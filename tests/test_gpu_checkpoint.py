"""Restart files through the C ABI (vh_save_checkpoint / vh_load_checkpoint):
a run resumed from a file continues bit for bit, in FP64 and in the mixed
mode, and a file of another grid is refused."""
import numpy as np
import pytest

from viral_b200 import _abi as A
from viral_b200 import configs as C
from viral_b200.hydro import Hydro

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [A.PREC_FP64, A.PREC_MIXED])
@pytest.mark.parametrize("boost_invariant", [True, False])
def test_resumed_run_continues_bit_for_bit(tmp_path, precision, boost_invariant):
    cfg = C.glauber_config(nx=40, ny=36, nz=1 if boost_invariant else 10, boost_invariant=boost_invariant,
                           precision=precision)
    path = str(tmp_path / "restart.bin")
    with C.make_hydro(cfg, C.glauber_inputs(cfg, b=5.0, seed=2)) as H:
        H.step(6)
        H.save_checkpoint(path)
        t_saved = H.tau
        H.step(6)
        ref, t_ref = H.get_state(), H.tau
    with Hydro(cfg) as R:
        assert R.load_checkpoint(path) == t_saved
        R.step(6)
        assert R.tau == t_ref
        assert np.array_equal(R.get_state(), ref)


def test_a_file_of_another_grid_is_refused(tmp_path):
    cfg = C.glauber_config(nx=20, ny=20, boost_invariant=True)
    path = str(tmp_path / "restart.bin")
    with C.make_hydro(cfg, C.glauber_inputs(cfg)) as H:
        H.save_checkpoint(path)
    other = C.glauber_config(nx=21, ny=20, boost_invariant=True)
    with Hydro(other) as R:
        with pytest.raises(A.VhError) as ex:
            R.load_checkpoint(path)
        assert ex.value.code == A.E_ARG and "grid" in str(ex.value)
    bad = tmp_path / "not_a_restart.bin"
    bad.write_bytes(b"\0" * 256)
    with Hydro(cfg) as R:
        with pytest.raises(A.VhError) as ex:
            R.load_checkpoint(str(bad))
        assert ex.value.code == A.E_ARG
