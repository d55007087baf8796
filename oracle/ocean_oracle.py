"""CPU oracle for the hydrostatic ocean-core time step (TEST INFRASTRUCTURE ONLY).

This module is the checker, never the product: only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg may import it.
The CUDA path in ``hydrostatic_ocean_core_benchmark_b200`` never routes through
it and fails loudly when its extension is missing.

It restates the reference's NumPy fp64 step (``libs/core/model3d_v05.py``
``Stepper3DV05``) and every operator on that path, in the same floating-point
operation order, so that its results are bit-identical to the reference. It is
pinned against golden vectors produced by the unmodified reference
(``tests/golden/make_golden.py``) and by the reference's own known answers
(TEOS-10 check value, ``tools/verify_v05.py:96-110``).

Two extensions that the reference lacks are expressed here as optional inputs,
each reducing bit-for-bit to the reference when given its special case:

* ``dzr``: a table of reference level thicknesses (stretched levels). ``None``
  gives the reference's uniform ``h_max / nz`` (``libs/core/domain.py:88``).
* ``taux_c``/``tauy_c``: a surface stress field at cell centres [N m-2]. ``None``
  gives the reference's scalar stress (``model3d_v05.py:176,355-356``). The
  u-face stress is the two-point average of the centre field, and the closure's
  u*^2 is ``hypot(taux_c, tauy_c) / rho0`` at each centre.

Layout is [k, j, i] (i fastest) fp64 throughout; interface arrays have nz+1
planes, interface 0 being the surface.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

# ----------------------------------------------------------------------------
# neighbour access on the periodic index layout (C-grid, reference grid.py:18-54)


def _east(a):
    """a[..., i+1] with periodic wrap."""
    return np.roll(a, -1, axis=-1)


def _west(a):
    """a[..., i-1] with periodic wrap."""
    return np.roll(a, 1, axis=-1)


def _north(a):
    """a[..., j+1, :] with periodic wrap."""
    return np.roll(a, -1, axis=-2)


def _south(a):
    """a[..., j-1, :] with periodic wrap."""
    return np.roll(a, 1, axis=-2)


def _shift(a, axis, by):
    return np.roll(a, by, axis=axis)


def inv_pos(a):
    """1/a where a > 0, else 0 (reference vertical_var.py:16-18, closure.py:39-40)."""
    return np.where(a > 0.0, 1.0 / np.where(a > 0.0, a, 1.0), 0.0)


# ----------------------------------------------------------------------------
# geometry: masks, partial cells, face thickness (reference domain.py:60-154)


class Geometry:
    """Domain geometry of the z-level coordinate.

    Follows ``Domain.__post_init__`` (domain.py:60-97), ``_face`` (:99-110),
    ``_resting_thickness`` (:113-129), ``face_thickness`` (:142-146) and
    ``depth_at_centres`` (:148-154). ``dzr`` optionally replaces the uniform
    reference thickness table.
    """

    def __init__(self, p, H, mask, dzr=None):
        nx, ny, nz = int(p.nx), int(p.ny), int(p.nz)
        self.nx, self.ny, self.nz = nx, ny, nz
        self.dx = p.lx / nx
        self.dy = p.ly / ny
        H = np.asarray(H, dtype=np.float64).reshape(ny, nx)
        mask = np.asarray(mask, dtype=np.float64).reshape(ny, nx)
        if p.bc_x not in ("periodic", "closed") or p.bc_y not in ("periodic", "closed"):
            raise ValueError("bc must be periodic|closed")
        if np.any(H[mask > 0] <= 0.0):
            raise ValueError("bathymetry must be positive in every wet cell")
        self.H, self.mask = H, mask
        self.face_rule = p.face_rule
        mu = mask * _east(mask)
        mv = mask * _north(mask)
        if p.bc_x != "periodic":
            mu[:, -1] = 0.0
        if p.bc_y != "periodic":
            mv[-1, :] = 0.0
        self.mask_u, self.mask_v = mu, mv
        self.h_max = float(np.max(H[mask > 0]))
        if dzr is None:
            dzr = np.full(nz, self.h_max / nz)
        self.dzr = np.asarray(dzr, dtype=np.float64).reshape(nz)
        edges = np.concatenate([[0.0], np.cumsum(self.dzr)])
        remaining = H[None, :, :] - edges[:-1, None, None]
        dz3 = np.clip(remaining, 0.0, self.dzr[:, None, None])
        thin = (dz3 > 0.0) & (dz3 < p.min_partial * self.dzr[:, None, None])
        dz3 = np.where(thin, 0.0, dz3)
        m3 = (dz3 > 0.0).astype(np.float64) * mask[None, :, :]
        self.dz3 = dz3 * m3
        self.mask3 = m3
        self.mask3u = self.mask3 * _east(self.mask3) * mu[None, :, :]
        self.mask3v = self.mask3 * _north(self.mask3) * mv[None, :, :]
        self.dz3u = self.mask3u * self.face(self.dz3, -1)
        self.dz3v = self.mask3v * self.face(self.dz3, -2)
        above = np.concatenate([np.zeros((1, ny, nx)), np.cumsum(self.dz3[:-1], axis=0)], axis=0)
        self.zc = above + 0.5 * self.dz3

    def face(self, a, axis):
        b = _shift(a, axis, -1)
        if self.face_rule == "min":
            return np.minimum(a, b)
        if self.face_rule == "mean":
            return 0.5 * (a + b)
        if self.face_rule == "harmonic":
            tot = a + b
            return np.where(tot > 0.0, 2.0 * a * b / np.where(tot > 0.0, tot, 1.0), 0.0)
        raise ValueError(f"face_rule must be min|mean|harmonic, got {self.face_rule!r}")


# ----------------------------------------------------------------------------
# vertical operators (reference vertical.py:17-44, vertical_var.py:21-145)


def thomas(sub, diag, sup, rhs):
    """Batched Thomas solve, one system per column (vertical.py:17-44)."""
    n = diag.shape[0]
    cs = np.empty_like(sup)
    ds = np.empty_like(rhs)
    cs[0] = sup[0] / diag[0]
    ds[0] = rhs[0] / diag[0]
    for k in range(1, n):
        den = diag[k] - sub[k] * cs[k - 1]
        cs[k] = sup[k] / den
        ds[k] = (rhs[k] - sub[k] * ds[k - 1]) / den
    x = np.empty_like(rhs)
    x[n - 1] = ds[n - 1]
    for k in range(n - 2, -1, -1):
        x[k] = ds[k] - cs[k] * x[k + 1]
    return x


def centre_spacing(dz3):
    """Interface spacing [nz+1] (vertical_var.py:21-32)."""
    nz = dz3.shape[0]
    out = np.empty((nz + 1,) + dz3.shape[1:])
    out[0] = dz3[0]
    out[1:nz] = 0.5 * (dz3[:nz - 1] + dz3[1:nz])
    out[nz] = dz3[nz - 1]
    return out


def _bottom_cells(mask3):
    below = np.concatenate([mask3[1:], np.zeros((1,) + mask3.shape[1:])], axis=0)
    return (mask3 > 0) & (below == 0)


def implicit_coeffs(K, dz3, dt, thv, drag, mask3):
    """Rows of A = I - thv dt Dz with dry identity rows (vertical_var.py:35-77)."""
    nz = K.shape[0] - 1
    dzi = centre_spacing(dz3)
    inv_dz = inv_pos(dz3)
    fac = thv * dt * inv_dz
    a_top = fac * K[:nz] * inv_pos(dzi[:nz])
    a_bot = fac * K[1:nz + 1] * inv_pos(dzi[1:nz + 1])
    sub = -a_top.copy()
    sup = -a_bot.copy()
    diag = 1.0 + a_top + a_bot
    diag[0] = 1.0 + a_bot[0]
    sub[0] = 0.0
    bottom = _bottom_cells(mask3)
    diag = np.where(bottom, 1.0 + a_top + thv * dt * drag * inv_dz, diag)
    sup = np.where(bottom, 0.0, sup)
    dry = mask3 == 0
    diag = np.where(dry, 1.0, diag)
    sub = np.where(dry, 0.0, sub)
    sup = np.where(dry, 0.0, sup)
    return sub, diag, sup


def explicit_diffusion(f, K, dz3, surf, drag, mask3):
    """Explicit Dz[f] with surface flux and cell drag (vertical_var.py:80-106)."""
    nz = f.shape[0]
    dzi = centre_spacing(dz3)
    flux = np.zeros((nz + 1,) + f.shape[1:])
    flux[1:nz] = K[1:nz] * (f[:nz - 1] - f[1:nz]) * inv_pos(dzi[1:nz])
    flux[0] = surf
    bottom = _bottom_cells(mask3)
    flux[1:nz] = np.where(bottom[:nz - 1], 0.0, flux[1:nz])
    flux[nz] = 0.0
    dragc = drag * f * bottom
    out = (flux[:nz] - flux[1:nz + 1]) * inv_pos(dz3)
    return (out - dragc * inv_pos(dz3)) * (mask3 > 0)


def w_from_transport(td):
    """w at interfaces from the layer-transport divergence (vertical_var.py:109-121)."""
    nz = td.shape[0]
    w = np.zeros((nz + 1,) + td.shape[1:])
    w[:nz] = -np.cumsum(td[::-1], axis=0)[::-1]
    return w


def buoyancy_potential(b, dz3):
    """Phi[k] = int_z^0 b dz' (vertical_var.py:132-136)."""
    above = np.concatenate([np.zeros((1,) + b.shape[1:]), np.cumsum((dz3 * b)[:-1], axis=0)], axis=0)
    return 0.5 * dz3 * b + above


def remove_thickness_mean(phi, dz3):
    """Phi minus its thickness-weighted column mean (vertical_var.py:139-145)."""
    total = np.sum(dz3, axis=0, keepdims=True)
    mean = np.sum(dz3 * phi, axis=0, keepdims=True) * inv_pos(total)
    return phi - mean


# ----------------------------------------------------------------------------
# masked C-grid operators (reference operators_masked.py:18-68)


def grad_x(eta, dx, mu):
    return mu * (_east(eta) - eta) / dx


def grad_y(eta, dy, mv):
    return mv * (_north(eta) - eta) / dy


def divergence(u, v, dx, dy, m):
    return m * ((u - _west(u)) / dx + (v - _south(v)) / dy)


def _wet_average(pairs):
    num = sum(w * f for f, w in pairs)
    den = sum(w for _, w in pairs)
    return np.where(den > 0.0, num / np.where(den > 0.0, den, 1.0), 0.0)


def v_at_u(v, mv, mu):
    """Coriolis average of v onto u points (operators_masked.py:45-52)."""
    vs, ms = _south(v), _south(mv)
    return _wet_average([(v, mv), (vs, ms), (_east(v), _east(mv)), (_east(vs), _east(ms))]) * mu


def u_at_v(u, mu, mv):
    """Coriolis average of u onto v points (operators_masked.py:55-61)."""
    uw, mw = _west(u), _west(mu)
    return _wet_average([(u, mu), (uw, mw), (_north(u), _north(mu)), (_north(uw), _north(mw))]) * mv


def hlaplacian(f, dx, dy, mu, mv, m):
    """D o G (operators_masked.py:64-68)."""
    return divergence(grad_x(f, dx, mu), grad_y(f, dy, mv), dx, dy, m)


# ----------------------------------------------------------------------------
# kappa = 1/3 / Superbee faces (reference advection_v06.py:21-108)

KAPPA = 1.0 / 3.0


def _superbee(r):
    return np.maximum(0.0, np.maximum(np.minimum(2.0 * r, 1.0), np.minimum(r, 2.0)))


def face_value(c, vel, axis, wet, limited):
    """Upwind-biased value on the face between c[i] and c[i+1] (advection_v06.py:21-47)."""
    cm = _shift(c, axis, 1)
    cp = _shift(c, axis, -1)
    cpp = _shift(c, axis, -2)
    if limited:
        d = cp - c
        eps = np.where(d == 0.0, 1.0, d)
        rp = np.where(d == 0.0, 0.0, (c - cm) / eps)
        rn = np.where(d == 0.0, 0.0, (cpp - cp) / eps)
        fp = c + 0.5 * _superbee(rp) * d
        fn = cp - 0.5 * _superbee(rn) * d
    else:
        fp = c + 0.25 * ((1.0 - KAPPA) * (c - cm) + (1.0 + KAPPA) * (cp - c))
        fn = cp - 0.25 * ((1.0 - KAPPA) * (cpp - cp) + (1.0 + KAPPA) * (cp - c))
    if wet is not None:
        fp = np.where(_shift(wet, axis, 1) > 0.0, fp, c)
        fn = np.where(_shift(wet, axis, -2) > 0.0, fn, cp)
    return np.where(vel > 0.0, fp, fn)


def face_value_z(c, w, wet3, limited):
    """Value on interior interfaces 1..nz-1, w positive upward (advection_v06.py:50-74)."""
    nz = c.shape[0]
    above, below = c[:-1], c[1:]
    pad = np.zeros_like(c[:1])
    far_up = np.concatenate([pad, c[:-2]], axis=0)
    far_dn = np.concatenate([c[2:], pad], axis=0)
    has_up = np.concatenate([np.zeros_like(wet3[:1]), wet3[:-2]], axis=0) > 0.0
    has_dn = np.concatenate([wet3[2:], np.zeros_like(wet3[:1])], axis=0) > 0.0
    d = above - below
    if limited:
        eps = np.where(d == 0.0, 1.0, d)
        ru = np.where(d == 0.0, 0.0, (below - far_dn) / eps)
        rd = np.where(d == 0.0, 0.0, (far_up - above) / eps)
        fu = below + 0.5 * _superbee(ru) * d
        fd = above - 0.5 * _superbee(rd) * d
    else:
        fu = below + 0.25 * ((1.0 - KAPPA) * (below - far_dn) + (1.0 + KAPPA) * (above - below))
        fd = above - 0.25 * ((1.0 - KAPPA) * (far_up - above) + (1.0 + KAPPA) * (above - below))
    fu = np.where(has_dn, fu, below)
    fd = np.where(has_up, fd, above)
    return np.where(w[1:nz] > 0.0, fu, fd)


def momentum_adv_up3(u, v, w, dx, dy, dz, m3u, m3v, limited):
    """Flux-form kappa-scheme momentum advection (advection_v06.py:77-108)."""
    nz = u.shape[0]
    ubar_c = 0.5 * (_west(u) + u)
    u_c = _west(face_value(u, _east(ubar_c), -1, m3u, limited))
    ax = (_east(ubar_c * u_c) - ubar_c * u_c) / dx
    vbar = 0.5 * (v + _east(v))
    fy = vbar * face_value(u, vbar, -2, m3u, limited)
    ay = (fy - _south(fy)) / dy
    wbar = 0.5 * (w + _east(w))
    fz = np.zeros_like(wbar)
    if nz > 1:
        fz[1:nz] = wbar[1:nz] * face_value_z(u, wbar, m3u, limited)
    az = (fz[:nz] - fz[1:nz + 1]) / dz
    vbar_c = 0.5 * (_south(v) + v)
    v_c = _south(face_value(v, _north(vbar_c), -2, m3v, limited))
    by = (_north(vbar_c * v_c) - vbar_c * v_c) / dy
    ubar = 0.5 * (u + _north(u))
    fx = ubar * face_value(v, ubar, -1, m3v, limited)
    bx = (fx - _west(fx)) / dx
    wbv = 0.5 * (w + _north(w))
    fzv = np.zeros_like(wbv)
    if nz > 1:
        fzv[1:nz] = wbv[1:nz] * face_value_z(v, wbv, m3v, limited)
    bz = (fzv[:nz] - fzv[1:nz + 1]) / dz
    return ax + ay + az, bx + by + bz


def momentum_adv_centred(u, v, w, dx, dy, dz):
    """Second-order centred flux-form momentum advection (advection.py:62-95)."""
    nz = u.shape[0]
    ubar_c = 0.5 * (_west(u) + u)
    ax = (_east(ubar_c) ** 2 - ubar_c ** 2) / dx
    vbar = 0.5 * (v + _east(v))
    uby = 0.5 * (u + _north(u))
    fy = vbar * uby
    ay = (fy - _south(fy)) / dy
    wbar = 0.5 * (w + _east(w))
    fz = np.zeros_like(wbar)
    if nz > 1:
        fz[1:nz] = wbar[1:nz] * 0.5 * (u[:-1] + u[1:])
    az = (fz[:nz] - fz[1:nz + 1]) / dz
    vbar_c = 0.5 * (_south(v) + v)
    by = (_north(vbar_c) ** 2 - vbar_c ** 2) / dy
    ubar = 0.5 * (u + _north(u))
    vbx = 0.5 * (v + _east(v))
    fx = ubar * vbx
    bx = (fx - _west(fx)) / dx
    wbv = 0.5 * (w + _north(w))
    fzv = np.zeros_like(wbv)
    if nz > 1:
        fzv[1:nz] = wbv[1:nz] * 0.5 * (v[:-1] + v[1:])
    bz = (fzv[:nz] - fzv[1:nz + 1]) / dz
    return ax + ay + az, bx + by + bz


# ----------------------------------------------------------------------------
# equation of state (reference eos.py:15-133). The polyTEOS10-bsq coefficients
# are Roquet et al. (2015) Table 4, the published values the reference uses.

_SEOS = (1.6550e-1, 7.6554e-1, 5.9520e-2, 7.4914e-4, 1.4970e-4, 1.1090e-5, 2.4341e-3)
_R0 = (4.6494977072e+01, -5.2099962525e+00, 2.2601900708e-01, 6.4326772569e-02,
       1.5616995503e-02, -1.7243708991e-03)
_C = dict(
    E000=8.0189615746e+02, E100=8.6672408165e+02, E200=-1.7864682637e+03, E300=2.0375295546e+03,
    E400=-1.2849161071e+03, E500=4.3227585684e+02, E600=-6.0579916612e+01,
    E010=2.6010145068e+01, E110=-6.5281885265e+01, E210=8.1770425108e+01, E310=-5.6888046321e+01,
    E410=1.7681814114e+01, E510=-1.9193502195e+00,
    E020=-3.7074170417e+01, E120=6.1548258127e+01, E220=-6.0362551501e+01, E320=2.9130021253e+01,
    E420=-5.4723692739e+00,
    E030=2.1661789529e+01, E130=-3.3449108469e+01, E230=1.9717078466e+01, E330=-3.1742946532e+00,
    E040=-8.3627885467e+00, E140=1.1311538584e+01, E240=-5.3563304045e+00,
    E050=5.4048723791e-01, E150=4.5111434961e-01, E060=-1.9098268277e-01,
    E001=1.9681925209e+01, E101=-4.2549998214e+01, E201=5.0774768218e+01, E301=-3.0938076334e+01,
    E401=6.6051753097e+00,
    E011=-1.3336301113e+01, E111=-4.4870114575e+00, E211=5.0042598061e+00, E311=-6.5399043664e-01,
    E021=6.7080479603e+00, E121=3.5063081279e+00, E221=-1.8795372996e+00,
    E031=-2.4649669534e+00, E131=-5.5077101279e-01, E041=5.5927935970e-01,
    E002=2.0660924175e+00, E102=-4.9527603989e+00, E202=2.5019633803e+00,
    E012=2.0564311499e+00, E112=-2.1311365518e-01, E022=-1.2419983026e+00,
    E003=-2.3342758797e-02, E103=-1.8507636718e-02, E013=3.7969820455e-01,
)
RDELTA_S = 32.0
R1_S0 = 0.875 / 35.16504
R1_T0 = 1.0 / 40.0
R1_Z0 = 1.0e-4


def rho_teos10(CT, SA, z):
    """polyTEOS10-bsq in-situ density, Horner form of eos.py:68-100."""
    c = _C
    r00, r01, r02, r03, r04, r05 = _R0
    zh = z * R1_Z0
    ss = np.sqrt((SA + RDELTA_S) * R1_S0)
    tt = CT * R1_T0
    r0 = (((((r05 * zh + r04) * zh + r03) * zh + r02) * zh + r01) * zh + r00) * zh
    rz3 = c["E013"] * tt + c["E103"] * ss + c["E003"]
    rz2 = ((c["E022"] * tt + c["E112"] * ss + c["E012"]) * tt
           + (c["E202"] * ss + c["E102"]) * ss + c["E002"])
    rz1 = ((((c["E041"] * tt + c["E131"] * ss + c["E031"]) * tt
             + (c["E221"] * ss + c["E121"]) * ss + c["E021"]) * tt
            + ((c["E311"] * ss + c["E211"]) * ss + c["E111"]) * ss + c["E011"]) * tt
           + (((c["E401"] * ss + c["E301"]) * ss + c["E201"]) * ss + c["E101"]) * ss
           + c["E001"])
    rz0 = ((((((c["E060"] * tt + c["E150"] * ss + c["E050"]) * tt
               + (c["E240"] * ss + c["E140"]) * ss + c["E040"]) * tt
              + ((c["E330"] * ss + c["E230"]) * ss + c["E130"]) * ss + c["E030"]) * tt
             + (((c["E420"] * ss + c["E320"]) * ss + c["E220"]) * ss + c["E120"]) * ss
             + c["E020"]) * tt
            + ((((c["E510"] * ss + c["E410"]) * ss + c["E310"]) * ss + c["E210"]) * ss
               + c["E110"]) * ss + c["E010"]) * tt
           + (((((c["E600"] * ss + c["E500"]) * ss + c["E400"]) * ss + c["E300"]) * ss
               + c["E200"]) * ss + c["E100"]) * ss + c["E000"])
    return ((rz3 * zh + rz2) * zh + rz1) * zh + rz0 + r0


def rho_anomaly(kind, T, S, z, rho0, alpha_T, beta_S, T0, S0):
    """Density anomaly (eos.py:103-127)."""
    if kind == "linear":
        return rho0 * (-alpha_T * (T - T0) + beta_S * (S - S0))
    if kind == "seos":
        a0, b0, lam1, lam2, mu1, mu2, nu_ts = _SEOS
        Ta, Sa = T - 10.0, S - 35.0
        return (-a0 * (1.0 + 0.5 * lam1 * Ta + mu1 * z) * Ta
                + b0 * (1.0 - 0.5 * lam2 * Sa - mu2 * z) * Sa
                - nu_ts * Ta * Sa)
    if kind == "teos10":
        return rho_teos10(T, S, z) - rho0
    raise ValueError(f"unknown eos {kind!r}")


def buoyancy(kind, T, S, z, g, rho0, alpha_T, beta_S, T0, S0):
    """b = -g rho' / rho0 (eos.py:130-133)."""
    return -g * rho_anomaly(kind, T, S, z, rho0, alpha_T, beta_S, T0, S0) / rho0


# ----------------------------------------------------------------------------
# TKE closure (reference closure.py:43-205)


def _column_geometry(dz3, mask3):
    nz = dz3.shape[0]
    zi = np.concatenate([np.zeros((1,) + dz3.shape[1:]), np.cumsum(dz3, axis=0)], axis=0)
    depth = zi[-1]
    d_bot = np.maximum(depth[None] - zi, 0.0)
    wet = np.zeros_like(zi)
    wet[1:nz] = mask3[:-1] * mask3[1:]
    return zi, d_bot, wet, centre_spacing(dz3)


def _budget_lengths(e, n2, dzi, z_s, z_b, wet, p):
    """Energy-budget mixing lengths of Gaspar et al. (1990) (closure.py:65-103)."""
    nz1 = e.shape[0]
    n2p = np.maximum(n2, 0.0)
    ek = np.maximum(e, p.e_min)
    out = {}
    for direction in ("up", "dn"):
        length = np.zeros_like(e)
        budget = ek.copy()
        for j in range(1, nz1):
            pad = np.zeros((j,) + e.shape[1:])
            if direction == "up":
                n2j = np.concatenate([pad, n2p[:-j]], axis=0)
                dzj = np.concatenate([pad, dzi[:-j]], axis=0)
            else:
                n2j = np.concatenate([n2p[j:], pad], axis=0)
                dzj = np.concatenate([dzi[j:], pad], axis=0)
            cost = n2j * dzj * (length + 0.5 * dzj)
            full = cost <= budget
            a = np.where(n2j > 0.0, n2j, 1.0)
            part = np.sqrt(np.maximum(length * length + 2.0 * budget / a, 0.0)) - length
            step = np.where(full, dzj, np.where(n2j > 0.0, np.clip(part, 0.0, dzj), dzj))
            new_len = length + np.where(budget > 0.0, step, 0.0)
            budget = np.where(full, budget - cost, 0.0)
            length = new_len
        out[direction] = length
    return (np.minimum(out["up"], z_s + p.z_0) * wet,
            np.minimum(out["dn"], z_b + p.z_0) * wet)


def _sweep_lengths(e, n2, dzi, z_s, z_b, wet, p):
    """Two-sweep limited buoyancy length (closure.py:106-129)."""
    nz1 = e.shape[0]
    n2c = np.maximum(n2, p.n2_min)
    ek = np.maximum(e, p.e_min)
    ell = np.sqrt(2.0 * ek / n2c)
    ell = np.minimum(ell, np.minimum(z_s + p.z_0, z_b + p.z_0))
    for k in range(1, nz1):
        ell[k] = np.minimum(ell[k], ell[k - 1] + dzi[k])
    for k in range(nz1 - 2, -1, -1):
        ell[k] = np.minimum(ell[k], ell[k + 1] + dzi[k + 1])
    ell = ell * wet
    return ell, ell


def tke_update(e, u, v, b, dz3, mask3, ustar2, dt, p, Km_old, Kh_old):
    """One TKE step; returns (e_new, K_m, K_h) on interfaces (closure.py:141-205)."""
    nz = dz3.shape[0]
    z_s, z_b, wet, dzi = _column_geometry(dz3, mask3)
    inv_dzi = inv_pos(dzi)
    uc = 0.5 * (u + _west(u))
    vc = 0.5 * (v + _south(v))
    du = np.zeros_like(e)
    dv = np.zeros_like(e)
    db = np.zeros_like(e)
    du[1:nz] = (uc[:-1] - uc[1:]) * inv_dzi[1:nz]
    dv[1:nz] = (vc[:-1] - vc[1:]) * inv_dzi[1:nz]
    db[1:nz] = (b[:-1] - b[1:]) * inv_dzi[1:nz]
    shear2 = (du ** 2 + dv ** 2) * wet
    n2 = db * wet
    if p.mxl == "recursive":
        l_up, l_dn = _sweep_lengths(e, n2, dzi, z_s, z_b, wet, p)
    elif p.mxl == "integral":
        l_up, l_dn = _budget_lengths(e, n2, dzi, z_s, z_b, wet, p)
    else:
        raise ValueError(f"unknown mixing length form {p.mxl!r}")
    l_k = np.maximum(p.l_min, np.sqrt(l_up * l_dn))
    l_eps = np.maximum(p.l_min, np.minimum(l_up, l_dn))
    prod = (Km_old - p.nu) * shear2 - (Kh_old - p.kappa) * n2
    diss = p.c_eps * np.sqrt(np.maximum(e, p.e_min)) / l_eps
    K_lay = 0.5 * (Km_old[:-1] + Km_old[1:])
    inv_dz3 = inv_pos(dz3)
    a_up = np.zeros_like(e)
    a_dn = np.zeros_like(e)
    a_up[1:nz] = dt * K_lay[:-1] * inv_dz3[:-1] * inv_dzi[1:nz]
    a_dn[1:nz] = dt * K_lay[1:] * inv_dz3[1:] * inv_dzi[1:nz]
    sub = -a_up
    sup = -a_dn
    diag = 1.0 + a_up + a_dn + dt * diss
    rhs = e + dt * prod
    e_surf = p.e_bb * ustar2
    bnd = wet <= 0.0
    diag = np.where(bnd, 1.0, diag)
    sub = np.where(bnd, 0.0, sub)
    sup = np.where(bnd, 0.0, sup)
    rhs = np.where(bnd, p.e_min, rhs)
    rhs[0] = np.where(mask3[0] > 0.0, e_surf, p.e_min)
    e_new = thomas(sub, diag, sup, rhs)
    e_new = np.maximum(e_new, p.e_min)
    e_new = np.where(wet > 0.0, e_new, p.e_min)
    e_new[0] = rhs[0]
    Km = p.c_k * l_k * np.sqrt(e_new) * wet + p.nu
    Kh = (Km - p.nu) / p.pr_t + p.kappa
    return e_new, Km, Kh


# ----------------------------------------------------------------------------
# variable-coefficient Helmholtz (reference solvers_var.py:22-197, solvers.py:145-148)


def _colours(ny, nx):
    j, i = np.indices((ny, nx))
    red = ((i + j) % 2 == 0)
    return red, ~red


class HelmOp:
    """A = I - c D[K G[.]] on one level (solvers_var.py:22-60)."""

    def __init__(self, nx, ny, lx, ly, coef, Ku, Kv, mask):
        self.nx, self.ny = nx, ny
        self.dx, self.dy = lx / nx, ly / ny
        self.coef = float(coef)
        self.Ku, self.Kv = np.ascontiguousarray(Ku), np.ascontiguousarray(Kv)
        self.mask = np.ascontiguousarray(mask)
        self.cx = self.coef * (1.0 / self.dx ** 2)
        self.cy = self.coef * (1.0 / self.dy ** 2)
        d = 1.0 + self.cx * (self.Ku + _west(self.Ku)) + self.cy * (self.Kv + _south(self.Kv))
        self.inv_diag = 1.0 / np.where(self.mask > 0, d, 1.0)

    def apply(self, x):
        x = x * self.mask
        fx = self.Ku * (_east(x) - x)
        fy = self.Kv * (_north(x) - x)
        lap = (fx - _west(fx)) / self.dx ** 2 + (fy - _south(fy)) / self.dy ** 2
        return (x - self.coef * lap) * self.mask + x * (1.0 - self.mask)

    def offdiag(self, x):
        return (self.cx * (self.Ku * _east(x) + _west(self.Ku) * _west(x))
                + self.cy * (self.Kv * _north(x) + _south(self.Kv) * _south(x)))


def gs_sweep(x, b, op, colours, reverse=False):
    """Red-black Gauss-Seidel sweep in place (solvers_var.py:63-69)."""
    for col in (colours[::-1] if reverse else colours):
        upd = op.inv_diag * (b + op.offdiag(x))
        x[col] = upd[col]
    x *= op.mask


class Helmholtz:
    """PCG-Jacobi / PCG-RBGS / RBGS / stationary multigrid (solvers_var.py:72-197)."""

    def __init__(self, nx, ny, lx, ly, coef, Ku, Kv, mask, kind, rtol, max_iter,
                 n_pre=2, n_post=2, min_size=8):
        if kind not in ("pcg_jacobi", "pcg_rbgs", "rbgs", "multigrid"):
            raise ValueError(f"unknown variable-coefficient solver {kind!r}")
        self.kind, self.rtol, self.max_iter = kind, rtol, max_iter
        self.nx, self.ny, self.lx, self.ly, self.coef = nx, ny, lx, ly, coef
        self.n_pre, self.n_post, self.min_size = n_pre, n_post, min_size
        self.mask = mask
        self.update(Ku, Kv)

    def update(self, Ku, Kv):
        self.op = HelmOp(self.nx, self.ny, self.lx, self.ly, self.coef, Ku, Kv, self.mask)
        self.colours = _colours(self.ny, self.nx)
        if self.kind == "multigrid":
            self.levels = [(self.op, self.colours)]
            op = self.op
            while (op.nx % 2 == 0 and op.ny % 2 == 0 and op.nx // 2 >= self.min_size
                   and op.ny // 2 >= self.min_size):
                cKu = 0.5 * (op.Ku[0::2, 1::2] + op.Ku[1::2, 1::2])
                cKv = 0.5 * (op.Kv[1::2, 0::2] + op.Kv[1::2, 1::2])
                cm = np.maximum.reduce([op.mask[0::2, 0::2], op.mask[0::2, 1::2],
                                        op.mask[1::2, 0::2], op.mask[1::2, 1::2]])
                op = HelmOp(op.nx // 2, op.ny // 2, self.lx, self.ly, self.coef, cKu, cKv, cm)
                self.levels.append((op, _colours(op.ny, op.nx)))

    def _vcycle(self, x, b, lvl):
        op, cols = self.levels[lvl]
        for _ in range(self.n_pre):
            gs_sweep(x, b, op, cols)
        if lvl + 1 < len(self.levels):
            r = (b - op.apply(x)) * op.mask
            cop = self.levels[lvl + 1][0]
            rc = 0.25 * (r[0::2, 0::2] + r[0::2, 1::2] + r[1::2, 0::2] + r[1::2, 1::2])
            e = self._vcycle(np.zeros((cop.ny, cop.nx)), rc, lvl + 1)
            x = x + np.repeat(np.repeat(e, 2, axis=0), 2, axis=1) * op.mask
        for _ in range(self.n_post):
            gs_sweep(x, b, op, cols, reverse=True)
        return x

    def _precond(self, r):
        if self.kind == "pcg_jacobi":
            return self.op.inv_diag * r
        z = np.zeros_like(r)
        gs_sweep(z, r, self.op, self.colours)
        gs_sweep(z, r, self.op, self.colours, reverse=True)
        return z

    def solve(self, rhs):
        """Returns (x, iterations, converged)."""
        rhs = rhs * self.op.mask
        norm_b = float(np.sqrt(np.sum(rhs * rhs)))
        x = np.zeros_like(rhs)
        if norm_b == 0.0:
            return x, 0, True
        tol = self.rtol * norm_b
        if self.kind in ("rbgs", "multigrid"):
            for it in range(1, self.max_iter + 1):
                if self.kind == "multigrid":
                    x = self._vcycle(x, rhs, 0)
                else:
                    gs_sweep(x, rhs, self.op, self.colours)
                res = float(np.sqrt(np.sum((rhs - self.op.apply(x)) ** 2)))
                if res <= tol:
                    return x, it, True
            return x, self.max_iter, False
        r = rhs.copy()
        z = self._precond(r)
        p = z.copy()
        rz = float(np.sum(r * z))
        for it in range(1, self.max_iter + 1):
            Ap = self.op.apply(p)
            alpha = rz / float(np.sum(p * Ap))
            x += alpha * p
            r -= alpha * Ap
            res = float(np.sqrt(np.sum(r * r)))
            if res <= tol:
                return x, it, True
            z = self._precond(r)
            rz_new = float(np.sum(r * z))
            p = z + (rz_new / rz) * p
            rz = rz_new
        return x, self.max_iter, False


# ----------------------------------------------------------------------------
# the step (reference model3d_v05.py:78-545)


@dataclass
class OracleState:
    """Prognostic state (reference model3d.py:34-47); e is None until the first TKE step."""

    u: np.ndarray
    v: np.ndarray
    b: np.ndarray
    eta: np.ndarray
    T: np.ndarray | None = None
    S: np.ndarray | None = None
    e: np.ndarray | None = None
    t: float = 0.0

    def copy(self):
        c = lambda a: None if a is None else np.array(a, copy=True)  # noqa: E731
        return OracleState(c(self.u), c(self.v), c(self.b), c(self.eta), c(self.T), c(self.S),
                           c(self.e), self.t)


class OracleStepper:
    """fp64 restatement of ``Stepper3DV05`` (model3d_v05.py:78-545).

    ``p`` is any object with the namelist attributes (nx, ny, nz, lx, ly, g,
    f0, h0, n2, nu, kappa, rho0, tau_x, tau_y, bottom_drag, scheme_name, theta,
    theta_cor, theta_v, n_picard, n_split, barotropic_average, solver_kind,
    rtol, max_iter, dt, bc_x, bc_y, face_rule, min_partial, eos, pgf,
    pgf_correction, advection, tracers, alpha_t, beta_s, t0, s0, cp, a_h, k_h,
    q_heat, q_salt, closure, mxl, c_k, c_eps, pr_t, z_0, e_min, l_min, e_bb,
    n2_min).
    """

    def __init__(self, p, H, mask, dzr=None, taux_c=None, tauy_c=None):
        if p.scheme_name not in ("fb", "theta", "split_explicit"):
            raise ValueError(f"unknown scheme {p.scheme_name!r}")
        if p.scheme_name == "theta" and not (0.0 < p.theta <= 1.0):
            raise ValueError("theta must lie in (0, 1]")
        if p.n_picard < 1:
            raise ValueError("n_picard must be >= 1")
        self.p = p
        self.geo = Geometry(p, H, mask, dzr)
        g = self.geo
        self.dt = float(p.dt)
        self.solver_iterations = 0
        self.solver_failures = 0
        self.solver_rebuilds = 0
        self.tridiagonal_solves = 0
        self.barotropic_substeps = 0
        self.solve_log: list[int] = []
        nz, ny, nx = g.nz, g.ny, g.nx
        self.Km = np.full((nz + 1, ny, nx), p.nu)
        self.Kh = np.full((nz + 1, ny, nx), p.kappa)
        self.dz_nom = p.h0 / nz
        # surface stress at u/v faces and the closure's u*^2
        if taux_c is None and tauy_c is None:
            self.tau_u = np.full((ny, nx), p.tau_x / p.rho0) * g.mask3u[0]
            self.tau_v = np.full((ny, nx), p.tau_y / p.rho0) * g.mask3v[0]
            self.ustar2 = np.full((ny, nx), np.hypot(p.tau_x, p.tau_y) / p.rho0)
        else:
            tx = np.zeros((ny, nx)) if taux_c is None else np.asarray(taux_c, float).reshape(ny, nx)
            ty = np.zeros((ny, nx)) if tauy_c is None else np.asarray(tauy_c, float).reshape(ny, nx)
            self.tau_u = (0.5 * (tx + _east(tx))) / p.rho0 * g.mask3u[0]
            self.tau_v = (0.5 * (ty + _north(ty))) / p.rho0 * g.mask3v[0]
            self.ustar2 = np.hypot(tx, ty) / p.rho0
        self.solver = None
        self._coefficients()
        if p.scheme_name == "split_explicit":
            c = np.sqrt(p.g * g.h_max)
            dt_baro = 1.0 / (c * np.sqrt(1.0 / g.dx ** 2 + 1.0 / g.dy ** 2))
            self.n_split = (p.n_split if p.n_split > 0
                            else max(1, int(np.ceil(1.2 * self.dt / dt_baro))))
            if self.dt / self.n_split > dt_baro:
                raise ValueError("barotropic substep above the gravity-wave limit")
        else:
            self.n_split = 0

    # -- coefficients (model3d_v05.py:141-167)
    def _coefficients(self):
        g, p = self.geo, self.p
        thv = p.theta_v
        self.tri_m = implicit_coeffs(self.Km, g.dz3, self.dt, thv, p.bottom_drag, g.mask3)
        self.tri_b = implicit_coeffs(self.Kh, g.dz3, self.dt, thv, 0.0, g.mask3)
        self.q = thomas(*self.tri_m, np.ones((g.nz, g.ny, g.nx)))
        self.tridiagonal_solves += 1
        qu = np.minimum(self.q, _east(self.q))
        qv = np.minimum(self.q, _north(self.q))
        self.Ku = np.sum(g.dz3u * qu, axis=0) * g.mask_u
        self.Kv = np.sum(g.dz3v * qv, axis=0) * g.mask_v
        if p.scheme_name == "theta":
            if self.solver is None:
                coef = p.g * p.theta ** 2 * self.dt ** 2
                self.solver = Helmholtz(g.nx, g.ny, p.lx, p.ly, coef, self.Ku, self.Kv, g.mask,
                                        p.solver_kind, p.rtol, p.max_iter)
            else:
                self.solver.update(self.Ku, self.Kv)
                self.solver_rebuilds += 1

    def _closure(self, s):
        g, p = self.geo, self.p
        e = s.e if s.e is not None else np.full((g.nz + 1, g.ny, g.nx), p.e_min)
        e_new, Km, Kh = tke_update(e, s.u, s.v, s.b, g.dz3, g.mask3, self.ustar2, self.dt, p,
                                   self.Km, self.Kh)
        self.Km, self.Kh = Km, Kh
        self.tridiagonal_solves += 1
        self._coefficients()
        return e_new

    def _pgf(self, b):
        """Common-depth pressure gradient (model3d_v05.py:195-230)."""
        g, p = self.geo, self.p
        phi = buoyancy_potential(b, g.dz3)
        if p.pgf == "remove":
            phi = remove_thickness_mean(phi, g.dz3)
        if not p.pgf_correction:
            return (grad_x(phi, g.dx, g.mask3u) * g.mask3u, grad_y(phi, g.dy, g.mask3v) * g.mask3v)
        zc = g.zc
        out = []
        for axis, fm, delta in ((-1, g.mask3u, g.dx), (-2, g.mask3v, g.dy)):
            phi_r, b_r, z_r = _shift(phi, axis, -1), _shift(b, axis, -1), _shift(zc, axis, -1)
            zf = 0.5 * (zc + z_r)
            left = phi + b * (zf - zc)
            right = phi_r + b_r * (zf - z_r)
            out.append(fm * (right - left) / delta)
        return out[0], out[1]

    def _w(self, u, v):
        g = self.geo
        return w_from_transport(divergence(g.dz3u * u, g.dz3v * v, g.dx, g.dy, g.mask3))

    def _column_solve(self, coeffs, rhs):
        self.tridiagonal_solves += 1
        return thomas(*coeffs, rhs)

    def _mom_extras(self, u, v, w):
        g, p = self.geo, self.p
        ex_u = np.zeros_like(u)
        ex_v = np.zeros_like(v)
        if p.advection in ("up3", "up3_tvd"):
            au, av = momentum_adv_up3(u, v, w, g.dx, g.dy, self.dz_nom, g.mask3u, g.mask3v,
                                      p.advection == "up3_tvd")
            ex_u -= au * g.mask3u
            ex_v -= av * g.mask3v
        elif p.advection != "none":
            au, av = momentum_adv_centred(u, v, w, g.dx, g.dy, self.dz_nom)
            ex_u -= au * g.mask3u
            ex_v -= av * g.mask3v
        if p.a_h > 0.0:
            ex_u += p.a_h * hlaplacian(u, g.dx, g.dy, g.mask3u, g.mask3v, g.mask3u)
            ex_v += p.a_h * hlaplacian(v, g.dx, g.dy, g.mask3u, g.mask3v, g.mask3v)
        return ex_u, ex_v

    def _div_bt(self, U, V):
        g = self.geo
        return divergence(U, V, g.dx, g.dy, g.mask)

    def _barotropic(self, U0, V0, eta, fx, fy):
        """Forward-backward substeps (model3d_v05.py:312-335)."""
        g, p = self.geo, self.p
        ddt = self.dt / self.n_split
        U, V, e = U0, V0, eta
        acc_u, acc_v = np.zeros_like(U0), np.zeros_like(V0)
        tc = p.theta_cor
        for _ in range(self.n_split):
            av_v, av_u = v_at_u(V, g.mask_v, g.mask_u), u_at_v(U, g.mask_u, g.mask_v)
            gxe = grad_x(e, g.dx, g.mask_u)
            gye = grad_y(e, g.dy, g.mask_v)
            Ui, Vi = U, V
            for _ in range(p.n_picard):
                v_cor = (1.0 - tc) * av_v + tc * v_at_u(Vi, g.mask_v, g.mask_u)
                u_cor = (1.0 - tc) * av_u + tc * u_at_v(Ui, g.mask_u, g.mask_v)
                Ui = (U + ddt * (p.f0 * v_cor - p.g * self.Ku * gxe + fx)) * g.mask_u
                Vi = (V + ddt * (-p.f0 * u_cor - p.g * self.Kv * gye + fy)) * g.mask_v
            U, V = Ui, Vi
            e = e - ddt * self._div_bt(U, V)
            acc_u += U
            acc_v += V
        self.barotropic_substeps += self.n_split
        if p.barotropic_average == "mean":
            return acc_u / self.n_split, acc_v / self.n_split, e
        return U, V, e

    def step(self, s: OracleState) -> OracleState:
        """One step (model3d_v05.py:337-415)."""
        g, p = self.geo, self.p
        dt, th, tc, thv = self.dt, p.theta, p.theta_cor, p.theta_v
        if p.scheme_name != "theta":
            th = 0.0
        e_new = self._closure(s) if p.closure == "tke" else s.e
        self._e_new = e_new
        m3 = g.mask3
        pgx, pgy = self._pgf(s.b)
        avp_v = v_at_u(s.v, g.mask3v, g.mask3u)
        avp_u = u_at_v(s.u, g.mask3u, g.mask3v)
        dzu_diff = explicit_diffusion(s.u, self.Km, g.dz3u, self.tau_u, p.bottom_drag, m3)
        dzv_diff = explicit_diffusion(s.v, self.Km, g.dz3v, self.tau_v, p.bottom_drag, m3)
        w_old = self._w(s.u, s.v)
        ex_u, ex_v = self._mom_extras(s.u, s.v, w_old)
        st_u = np.zeros((g.nz, g.ny, g.nx))
        st_v = np.zeros((g.nz, g.ny, g.nx))
        st_u[0] = thv * dt * self.tau_u * inv_pos(g.dz3u[0])
        st_v[0] = thv * dt * self.tau_v * inv_pos(g.dz3v[0])
        st_u = st_u + dt * ex_u
        st_v = st_v + dt * ex_v
        if p.scheme_name == "split_explicit":
            return self._step_split(s, pgx, pgy, avp_u, avp_v, dzu_diff, dzv_diff, st_u, st_v)
        gx_eta = grad_x(s.eta, g.dx, g.mask_u)[None] * g.mask3u
        gy_eta = grad_y(s.eta, g.dy, g.mask_v)[None] * g.mask3v
        div_old = self._div_bt(np.sum(g.dz3u * s.u, axis=0), np.sum(g.dz3v * s.v, axis=0))
        u_it, v_it, eta_new = s.u, s.v, s.eta
        for _ in range(p.n_picard):
            v_cor = (1.0 - tc) * avp_v + tc * v_at_u(v_it, g.mask3v, g.mask3u)
            u_cor = (1.0 - tc) * avp_u + tc * u_at_v(u_it, g.mask3u, g.mask3v)
            gu = (s.u + dt * (p.f0 * v_cor + pgx) - p.g * dt * (1.0 - th) * gx_eta
                  + (1.0 - thv) * dt * dzu_diff)
            gv = (s.v + dt * (-p.f0 * u_cor + pgy) - p.g * dt * (1.0 - th) * gy_eta
                  + (1.0 - thv) * dt * dzv_diff)
            gh_u = self._column_solve(self.tri_m, gu + st_u) * m3
            gh_v = self._column_solve(self.tri_m, gv + st_v) * m3
            if p.scheme_name == "theta":
                div_g = self._div_bt(np.sum(g.dz3u * gh_u, axis=0), np.sum(g.dz3v * gh_v, axis=0))
                rhs = s.eta - dt * ((1.0 - th) * div_old + th * div_g)
                eta_new, its, ok = self.solver.solve(rhs)
                self.solver_iterations += its
                self.solver_failures += 0 if ok else 1
                self.solve_log.append(its)
                u_it = gh_u - p.g * dt * th * self.q * grad_x(eta_new, g.dx, g.mask_u)[None] * g.mask3u
                v_it = gh_v - p.g * dt * th * self.q * grad_y(eta_new, g.dy, g.mask_v)[None] * g.mask3v
                u_it, v_it = u_it * m3, v_it * m3
            else:
                u_it, v_it = gh_u, gh_v
        if p.scheme_name == "fb":
            eta_new = s.eta - dt * self._div_bt(np.sum(g.dz3u * u_it, axis=0),
                                                np.sum(g.dz3v * v_it, axis=0))
        w = self._w(u_it, v_it)
        return self._tracers(s, u_it, v_it, w, eta_new)

    def _step_split(self, s, pgx, pgy, avp_u, avp_v, dzu_diff, dzv_diff, st_u, st_v):
        """Split-explicit step (model3d_v05.py:417-463)."""
        g, p = self.geo, self.p
        dt, tc, thv = self.dt, p.theta_cor, p.theta_v
        m3 = g.mask3
        U0 = np.sum(g.dz3u * s.u, axis=0)
        V0 = np.sum(g.dz3v * s.v, axis=0)
        u_it, v_it = s.u, s.v
        gh_u = gh_v = None
        for _ in range(p.n_picard):
            v_cor = (1.0 - tc) * avp_v + tc * v_at_u(v_it, g.mask3v, g.mask3u)
            u_cor = (1.0 - tc) * avp_u + tc * u_at_v(u_it, g.mask3u, g.mask3v)
            gu = s.u + dt * (p.f0 * v_cor + pgx) + (1.0 - thv) * dt * dzu_diff
            gv = s.v + dt * (-p.f0 * u_cor + pgy) + (1.0 - thv) * dt * dzv_diff
            gh_u = self._column_solve(self.tri_m, gu + st_u) * m3
            gh_v = self._column_solve(self.tri_m, gv + st_v) * m3
            u_it, v_it = gh_u, gh_v
        Um, Vm = np.sum(g.dz3u * gh_u, axis=0), np.sum(g.dz3v * gh_v, axis=0)
        cor_x = p.f0 * ((1.0 - tc) * v_at_u(V0, g.mask_v, g.mask_u) + tc * v_at_u(Vm, g.mask_v, g.mask_u))
        cor_y = -p.f0 * ((1.0 - tc) * u_at_v(U0, g.mask_u, g.mask_v) + tc * u_at_v(Um, g.mask_u, g.mask_v))
        fx = (Um - U0) / dt - cor_x
        fy = (Vm - V0) / dt - cor_y
        U, V, eta_new = self._barotropic(U0, V0, s.eta, fx, fy)
        Hu = np.sum(g.dz3u, axis=0)
        Hv = np.sum(g.dz3v, axis=0)
        ihu = inv_pos(Hu)
        ihv = inv_pos(Hv)
        u_new = (gh_u - np.sum(g.dz3u * gh_u, axis=0) * ihu + U * ihu) * g.mask3u
        v_new = (gh_v - np.sum(g.dz3v * gh_v, axis=0) * ihv + V * ihv) * g.mask3v
        w = self._w(u_new, v_new)
        return self._tracers(s, u_new, v_new, w, eta_new)

    def _tracer_adv(self, c, u, v, w):
        """Flux-form tracer advection (model3d_v05.py:482-512)."""
        g, p = self.geo, self.p
        scheme = p.advection
        if scheme == "centered2":
            cx = 0.5 * (c + _east(c))
            cy = 0.5 * (c + _north(c))
        elif scheme in ("up3", "up3_tvd"):
            cx = face_value(c, u, -1, g.mask3, scheme == "up3_tvd")
            cy = face_value(c, v, -2, g.mask3, scheme == "up3_tvd")
        else:
            cx = np.where(u > 0, c, _east(c))
            cy = np.where(v > 0, c, _north(c))
        fx = g.dz3u * u * cx
        fy = g.dz3v * v * cy
        inv = inv_pos(g.dz3)
        hdiv = ((fx - _west(fx)) / g.dx + (fy - _south(fy)) / g.dy) * inv
        nz = c.shape[0]
        cf = np.zeros((nz + 1,) + c.shape[1:])
        if scheme in ("up3", "up3_tvd"):
            cf[1:nz] = face_value_z(c, w, g.mask3, scheme == "up3_tvd")
        else:
            cf[1:nz] = 0.5 * (c[:nz - 1] + c[1:nz])
        cf[0] = c[0]
        vdiv = (w[:nz] * cf[:nz] - w[1:] * cf[1:]) * inv
        return (hdiv + vdiv) * g.mask3

    def _tracer(self, c, u, v, w, surf, source=None):
        """One tracer (model3d_v05.py:466-480)."""
        g, p, dt = self.geo, self.p, self.dt
        thv = p.theta_v
        tend = np.zeros_like(c) if source is None else source
        if p.advection != "none":
            tend = tend - self._tracer_adv(c, u, v, w)
        if p.k_h > 0.0:
            tend = tend + p.k_h * hlaplacian(c, g.dx, g.dy, g.mask3u, g.mask3v, g.mask3)
        rhs = c + dt * tend + (1.0 - thv) * dt * explicit_diffusion(c, self.Kh, g.dz3, surf, 0.0, g.mask3)
        rhs[0] = rhs[0] + thv * dt * surf * inv_pos(g.dz3[0])
        return self._column_solve(self.tri_b, rhs) * g.mask3

    def _tracers(self, s, u, v, w, eta_new):
        """Tracers and the equation of state (model3d_v05.py:514-533)."""
        g, p, dt = self.geo, self.p, self.dt
        if p.tracers == "TS":
            fT = np.full((g.ny, g.nx), p.q_heat / (p.rho0 * p.cp))
            fS = np.full((g.ny, g.nx), p.q_salt)
            T_new = self._tracer(s.T, u, v, w, fT)
            S_new = self._tracer(s.S, u, v, w, fS)
            b_new = buoyancy(p.eos, T_new, S_new, g.zc, p.g, p.rho0, p.alpha_t, p.beta_s,
                             p.t0, p.s0) * g.mask3
            return OracleState(u, v, b_new, eta_new, T_new, S_new, self._e_new, s.t + dt)
        source = -p.n2 * (0.5 * (w[:-1] + w[1:]))
        b_new = self._tracer(s.b, u, v, w, np.zeros((g.ny, g.nx)), source=source)
        return OracleState(u, v, b_new, eta_new, None, None, self._e_new, s.t + dt)

    def integrate(self, s: OracleState, n_steps: int) -> OracleState:
        for _ in range(n_steps):
            s = self.step(s)
        return s


# ----------------------------------------------------------------------------
# the gate's error metric (reference tools/compare_backends3d.py:52-67)


def field_error(a, b, state_scale):
    """Relative L2, or L2 relative to the state scale for a near-zero field."""
    num = float(np.sqrt(np.sum((a - b) ** 2)))
    den = float(np.sqrt(np.sum(b * b)))
    if den > 1e-11 * state_scale:
        return num / den
    return num / state_scale if state_scale > 0.0 else num
