"""Re-exports the case definitions of tests/golden/make_golden.py."""
import os
import sys

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
from make_golden import (aerosol_case, aero_channels, band_case, emitters_case, headline_case,
                         ice_depth2_case, scattering_point_case, aerosol_jacobian_case, curtain_ctl,  # noqa: E402,F401
                         curtain_jacobian_case, curtain_scattering_case, fov_case,
                         jacobian_case, mixed_case, tables_digest)
