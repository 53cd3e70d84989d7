"""The oracle's direct quadrature where the lognormal MOR lies far outside the
lam_t domain: its renormalisation D = Phi(b) - Phi(a) underflows FP64 (mu
about 38 sigma or more below ln lam_t_lo) and the oracle takes the density
exp(-d^2 / 2) / D in logs, so the counts stay finite and continuous in sigma
across the switch."""
import numpy as np
import pytest

import oracle as O
from y3_cluster_cpp_b200 import synthetic


def _counts(sigma, lam_t=(44.7, 1000.0)):
    g = synthetic.grid(1, lam_t_lo=lam_t[0], lam_t_hi=lam_t[1])
    p = synthetic.fiducial()
    p.sigma = sigma
    pz, pc = synthetic.plob_baseline()
    c, _, _ = O.direct_eval(g, pz, pc, p.mor, O.cosmo(p.om, p.h0), p.tables)
    return c


@pytest.mark.parametrize("sigma", [0.09, 0.07, 0.05])
def test_direct_eval_finite_where_the_mor_normalisation_underflows(sigma):
    c = _counts(sigma)
    assert np.all(np.isfinite(c)) and np.all(c > 0)


def test_direct_eval_continuous_across_the_log_switch():
    # sigma from 0.106 to 0.096 moves the lowest-mass cells' D through the
    # 1e-280 switch (mu about 36 sigma below ln 44.7); the counts move
    # smoothly, with no jump between neighbouring sigmas.
    s = np.linspace(0.106, 0.096, 11)
    c = np.array([_counts(x) for x in s])
    d = np.diff(c, axis=0)
    dd = np.diff(d, axis=0)
    assert np.all(np.abs(dd) <= 0.05 * np.abs(d).max(axis=0) + 1e-12)
