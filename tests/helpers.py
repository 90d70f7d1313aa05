"""Comparison helpers shared by the parity tests."""
import numpy as np

C1 = 1.19104259e-8
C2 = 1.43877506


def brightness(rad, nu):
    """Brightness temperature (src/forwardmodel.c:7-11), vectorised."""
    nu = np.asarray(nu, dtype=np.float64)
    return C2 * nu / np.log1p(C1 * nu ** 3 / np.asarray(rad, dtype=np.float64))


def bt_error(rad, rad_ref, nus):
    """Max |BT - BT_ref| in K over finite, positive radiances."""
    nus = np.asarray(nus)[None, :]
    ok = np.isfinite(rad_ref) & (rad_ref > 0)
    if not ok.any():
        return 0.0
    d = np.abs(brightness(np.where(ok, rad, 1.0), nus) - brightness(np.where(ok, rad_ref, 1.0), nus))
    return float(np.max(np.where(ok, d, 0.0)))


def max_rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    den = np.maximum(np.abs(b), 1e-300)
    return float(np.max(np.abs(a - b) / den))
