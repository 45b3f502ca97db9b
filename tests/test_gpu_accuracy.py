"""FP16 deviation storage against FP64 on the GPU (lbm_porouschem_b200.accuracy): the
errors in velocity, temperature, permeability and conversion-front position stay within
the stated bounds."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_front_position_helper():
    alpha = np.ones((10, 4))
    alpha[:3] = 0.0                      # converted up to x = 2
    alpha[3] = 0.6                       # conversion 0.4 at x = 3
    react = np.ones((10, 4), dtype=bool)
    from lbm_porouschem_b200.accuracy import front_position
    assert front_position(alpha, react) == pytest.approx(2 + 0.5 / 0.6)


def test_fp16_front_and_fields():
    from lbm_porouschem_b200.accuracy import front_case
    r = front_case(128, 48, seed=3, steps=3000)
    print(r)
    assert r["cells_converted_fp64"] > 20
    assert r["solid_cells_differing"] <= 2
    assert r["front_dx_cells"] <= 1.0
    # a slow (|u| ~ 2e-4) transient: FP16 keeps ~11 bits of each deviation, so the
    # velocity carries ~15 % and the temperature ~4 % relative L2 error (256 x 64 case)
    assert r["u_rel_l2"] < 0.3
    assert r["T_rel_l2"] < 0.1


def test_fp16_permeability():
    from lbm_porouschem_b200.accuracy import permeability_case
    r = permeability_case(64, 32, seed=2, steps=4000)
    print(r)
    assert r["k_rel_diff"] < 1e-2        # 1.5e-3 at 128 x 64
