"""Frozen Costanzi-2026 projection-effect EMG coefficient table.

The eight coefficients (a_tau, b_tau, a_mu, b_mu, a_sig, b_sig, a_fprj,
b_fprj) of P(lambda_obs | lambda_true, z) on a fixed 15-node redshift grid
spanning [0.10, 0.80].  These numbers are calibration data that must be
identical to the reference's table (y3_buzzard/prj_params.py:28-55) for the
selection function to be a drop-in; they are evaluated as linear splines in z
with constant extrapolation (prj_params.py:122-130).

``baseline_constant_table()`` gives the z-independent coefficients of the
synthetic benchmark kernel: Gaussian sigma = 0.1 lambda_t with a projection
tail of weight 0.1 and rate tau = b_tau / lambda_t^a_tau taken at z = 0.45.
"""
from __future__ import annotations

import numpy as np

COEFF_NAMES = ("a_tau", "b_tau", "a_mu", "b_mu", "a_sig", "b_sig", "a_fprj", "b_fprj")

Z = np.array([0.1, 0.15000000000000002, 0.2, 0.25, 0.30000000000000004, 0.35, 0.4,
              0.45000000000000007, 0.5, 0.55, 0.6, 0.65, 0.7000000000000001, 0.75, 0.8])

TABLE = {
    "a_tau": [0.442166204, 0.518481914, 0.568603921, 0.477236476, 0.520278762,
              0.579677963, 0.555190684, 0.672770912, 0.478623398, 0.549620102,
              0.480748319, 0.578522658, 0.671535976, 0.505164749, 0.58955537],
    "b_tau": [1.18217964, 1.47500549, 2.02559386, 1.38676832, 1.32616774,
              1.67202719, 1.51274293, 1.95006009, 1.18386488, 1.36976846,
              1.05592613, 1.30622288, 1.86155835, 1.11381729, 1.55322604],
    "a_mu": [-0.364318121, -0.23432317, -0.656963951, -0.922603116, -0.846333985,
             -1.08055911, -1.18280131, -1.06499383, -1.39776432, -1.73727975,
             -1.89795303, -2.06646039, -2.11221354, -2.33692459, -2.68990643],
    "b_mu": [1.05327406, 1.02863546, 1.00438937, 1.02999661, 1.07731829,
             1.00753429, 1.02754167, 0.984235605, 1.0482203, 1.04839327,
             1.0613957, 1.06299404, 1.07220168, 1.06769774, 1.17169173],
    "a_sig": [0.426034095, 0.399889486, 0.36483048, 0.400337495, 0.412239723,
              0.352441888, 0.386464927, 0.346387159, 0.36257126, 0.414359103,
              0.396064175, 0.392899807, 0.412642261, 0.411313571, 0.516942252],
    "b_sig": [1.03790465, 1.07103564, 1.19439168, 1.15625107, 1.21959668,
              1.36154101, 1.29767428, 1.38632059, 1.37829562, 1.1874275,
              1.33730986, 1.43217579, 1.36804085, 1.49303631, 1.25987859],
    "a_fprj": [9.77919696, 9.84852044, 9.85900036, 9.66653259, 9.80163756,
               9.57966267, 9.89274466, 9.53433063, 8.20542109, 9.93404856,
               9.89089118, 7.86185779, 8.44425519, 8.33876275, 9.83602795],
    "b_fprj": [0.259342564, 0.392345959, 0.938787218, 0.76558764, 0.438594201,
               0.987913546, 0.819593953, 0.996036691, 0.906686505, 0.997565086,
               0.99306453, 0.984970784, 0.951840743, 0.987248745, 0.832798309],
}


def default_table():
    """(z [15], coef [8, 15]) of the reference's frozen table."""
    return Z.copy(), np.array([TABLE[k] for k in COEFF_NAMES], dtype=np.float64)


def baseline_constant_table(sigma_frac=0.1, f_prj=0.1, z_tau=0.45):
    """Constant-in-z coefficients for the synthetic P(lambda_o | lambda_t):
    mu = lambda_t, sigma = sigma_frac lambda_t, tau = b_tau lambda_t^-a_tau
    (reference coefficients at z_tau), f_prj constant."""
    i = int(np.argmin(np.abs(Z - z_tau)))
    z = np.array([0.0, 2.0])
    vals = {"a_tau": TABLE["a_tau"][i], "b_tau": TABLE["b_tau"][i],
            "a_mu": 0.0, "b_mu": 1.0, "a_sig": 1.0, "b_sig": sigma_frac,
            "a_fprj": 0.0, "b_fprj": f_prj}
    coef = np.array([[vals[k], vals[k]] for k in COEFF_NAMES], dtype=np.float64)
    return z, coef
