"""The equation of state on the host, for initial states written to bundles.

b = -g rho'(T, S, z) / rho0 with the linear EOS, the S-EOS or polyTEOS10-bsq
(reference libs/core/eos.py:68-133; the polyTEOS10-bsq and S-EOS coefficient
tables are Roquet et al. 2015's published values). The operations and their
order are those of the device EOS (csrc/oc_internal.cuh rho_teos10_n /
rho_anomaly_n), which NumPy evaluates without contraction, so a state built
here carries the b the step itself would diagnose.
"""

from __future__ import annotations

import numpy as np


def rho_teos10(CT, SA, z):
    zh = z * 1.0e-4
    ss = np.sqrt((SA + 32.0) * (0.875 / 35.16504))
    tt = CT * (1.0 / 40.0)
    r0 = (((((-1.7243708991e-03 * zh + 1.5616995503e-02) * zh + 6.4326772569e-02) * zh
            + 2.2601900708e-01) * zh + -5.2099962525e+00) * zh + 4.6494977072e+01) * zh
    rz3 = 3.7969820455e-01 * tt + -1.8507636718e-02 * ss + -2.3342758797e-02
    rz2 = ((-1.2419983026e+00 * tt + -2.1311365518e-01 * ss + 2.0564311499e+00) * tt
           + (2.5019633803e+00 * ss + -4.9527603989e+00) * ss + 2.0660924175e+00)
    rz1 = ((((5.5927935970e-01 * tt + -5.5077101279e-01 * ss + -2.4649669534e+00) * tt
             + (-1.8795372996e+00 * ss + 3.5063081279e+00) * ss + 6.7080479603e+00) * tt
            + ((-6.5399043664e-01 * ss + 5.0042598061e+00) * ss + -4.4870114575e+00) * ss
            + -1.3336301113e+01) * tt
           + (((6.6051753097e+00 * ss + -3.0938076334e+01) * ss + 5.0774768218e+01) * ss
              + -4.2549998214e+01) * ss
           + 1.9681925209e+01)
    rz0 = ((((((-1.9098268277e-01 * tt + 4.5111434961e-01 * ss + 5.4048723791e-01) * tt
               + (-5.3563304045e+00 * ss + 1.1311538584e+01) * ss + -8.3627885467e+00) * tt
              + ((-3.1742946532e+00 * ss + 1.9717078466e+01) * ss + -3.3449108469e+01) * ss
              + 2.1661789529e+01) * tt
             + (((-5.4723692739e+00 * ss + 2.9130021253e+01) * ss + -6.0362551501e+01) * ss
                + 6.1548258127e+01) * ss
             + -3.7074170417e+01) * tt
            + ((((-1.9193502195e+00 * ss + 1.7681814114e+01) * ss + -5.6888046321e+01) * ss
                + 8.1770425108e+01) * ss
               + -6.5281885265e+01) * ss
            + 2.6010145068e+01) * tt
           + (((((-6.0579916612e+01 * ss + 4.3227585684e+02) * ss + -1.2849161071e+03) * ss
                + 2.0375295546e+03) * ss
               + -1.7864682637e+03) * ss
              + 8.6672408165e+02) * ss
           + 8.0189615746e+02)
    return ((rz3 * zh + rz2) * zh + rz1) * zh + rz0 + r0


def rho_anomaly(p, T, S, z):
    if p.eos == "linear":
        return p.rho0 * (-p.alpha_t * (T - p.t0) + p.beta_s * (S - p.s0))
    if p.eos == "seos":
        Ta, Sa = T - 10.0, S - 35.0
        return (-1.6550e-1 * (1.0 + (0.5 * 5.9520e-2) * Ta + 1.4970e-4 * z) * Ta
                + 7.6554e-1 * (1.0 - (0.5 * 7.4914e-4) * Sa - 1.1090e-5 * z) * Sa
                - 2.4341e-3 * Ta * Sa)
    if p.eos == "teos10":
        return rho_teos10(T, S, z) - p.rho0
    raise ValueError(f"unknown eos {p.eos!r}")


def buoyancy(p, T, S, z):
    return -p.g * rho_anomaly(p, T, S, z) / p.rho0
