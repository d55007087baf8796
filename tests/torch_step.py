"""Float64 torch restatement of the ocean step, differentiable by torch.autograd.

Test infrastructure: the reference gradient that pins the hand-written adjoint
(``oc_adjoint_step``). It restates the oracle (``oracle/ocean_oracle.py``, which
follows reference ``libs/core/model3d_v05.py:337-533``) function by function in
torch for the configuration the adjoint covers: the theta scheme with TS
tracers, constant viscosity and diffusivity (closure none), kappa / TVD / centred
advection, any EOS, the common-depth pressure gradient, a surface-stress field
and stretched levels. The Helmholtz solve is PCG-Jacobi to rtol 1e-15 inside an
autograd function whose backward is the solve with the same (symmetric)
operator, so its forward agrees with the oracle's rtol-1e-12 solve to that
tolerance, not bit for bit.
"""

from __future__ import annotations

import torch

from oracle import ocean_oracle as orc

KAPPA = 1.0 / 3.0


def _t(a, dev):
    return torch.as_tensor(a, dtype=torch.float64, device=dev)


def east(a):
    return torch.roll(a, -1, -1)


def west(a):
    return torch.roll(a, 1, -1)


def north(a):
    return torch.roll(a, -1, -2)


def south(a):
    return torch.roll(a, 1, -2)


def shift(a, axis, by):
    return torch.roll(a, by, axis)


def thomas(sub, diag, sup, rhs):
    n = diag.shape[0]
    cs = [sup[0] / diag[0]]
    ds = [rhs[0] / diag[0]]
    for k in range(1, n):
        den = diag[k] - sub[k] * cs[k - 1]
        cs.append(sup[k] / den)
        ds.append((rhs[k] - sub[k] * ds[k - 1]) / den)
    x = [None] * n
    x[n - 1] = ds[n - 1]
    for k in range(n - 2, -1, -1):
        x[k] = ds[k] - cs[k] * x[k + 1]
    return torch.stack(x)


def superbee(r):
    z = torch.zeros_like(r)
    return torch.maximum(z, torch.maximum(torch.clamp(2.0 * r, max=1.0), torch.clamp(r, max=2.0)))


def face_value(c, vel, axis, wet, limited):
    cm, cp, cpp = shift(c, axis, 1), shift(c, axis, -1), shift(c, axis, -2)
    if limited:
        d = cp - c
        zero = d == 0.0
        eps = torch.where(zero, torch.ones_like(d), d)
        rp = torch.where(zero, torch.zeros_like(d), (c - cm) / eps)
        rn = torch.where(zero, torch.zeros_like(d), (cpp - cp) / eps)
        fp = c + 0.5 * superbee(rp) * d
        fn = cp - 0.5 * superbee(rn) * d
    else:
        fp = c + 0.25 * ((1.0 - KAPPA) * (c - cm) + (1.0 + KAPPA) * (cp - c))
        fn = cp - 0.25 * ((1.0 - KAPPA) * (cpp - cp) + (1.0 + KAPPA) * (cp - c))
    if wet is not None:
        fp = torch.where(shift(wet, axis, 1) > 0.0, fp, c)
        fn = torch.where(shift(wet, axis, -2) > 0.0, fn, cp)
    return torch.where(vel > 0.0, fp, fn)


def face_value_z(c, w, wet3, limited):
    nz = c.shape[0]
    above, below = c[:-1], c[1:]
    pad = torch.zeros_like(c[:1])
    far_up = torch.cat([pad, c[:-2]], 0)
    far_dn = torch.cat([c[2:], pad], 0)
    has_up = torch.cat([torch.zeros_like(wet3[:1]), wet3[:-2]], 0) > 0.0
    has_dn = torch.cat([wet3[2:], torch.zeros_like(wet3[:1])], 0) > 0.0
    d = above - below
    if limited:
        zero = d == 0.0
        eps = torch.where(zero, torch.ones_like(d), d)
        ru = torch.where(zero, torch.zeros_like(d), (below - far_dn) / eps)
        rd = torch.where(zero, torch.zeros_like(d), (far_up - above) / eps)
        fu = below + 0.5 * superbee(ru) * d
        fd = above - 0.5 * superbee(rd) * d
    else:
        fu = below + 0.25 * ((1.0 - KAPPA) * (below - far_dn) + (1.0 + KAPPA) * (above - below))
        fd = above - 0.25 * ((1.0 - KAPPA) * (far_up - above) + (1.0 + KAPPA) * (above - below))
    fu = torch.where(has_dn, fu, below)
    fd = torch.where(has_up, fd, above)
    return torch.where(w[1:nz] > 0.0, fu, fd)


def zpad(inner, nz):
    """(nz+1) interface array with zero top and bottom around rows 1..nz-1."""
    z = torch.zeros_like(inner[:1])
    return torch.cat([z, inner, z], 0) if nz > 1 else torch.cat([z, z], 0)


def momentum_adv(u, v, w, dx, dy, dz, m3u, m3v, scheme):
    nz = u.shape[0]
    if scheme in ("up3", "up3_tvd"):
        lim = scheme == "up3_tvd"
        ubar_c = 0.5 * (west(u) + u)
        u_c = west(face_value(u, east(ubar_c), -1, m3u, lim))
        ax = (east(ubar_c * u_c) - ubar_c * u_c) / dx
        vbar = 0.5 * (v + east(v))
        fy = vbar * face_value(u, vbar, -2, m3u, lim)
        ay = (fy - south(fy)) / dy
        wbar = 0.5 * (w + east(w))
        fz = zpad(wbar[1:nz] * face_value_z(u, wbar, m3u, lim), nz)
        az = (fz[:nz] - fz[1:nz + 1]) / dz
        vbar_c = 0.5 * (south(v) + v)
        v_c = south(face_value(v, north(vbar_c), -2, m3v, lim))
        by = (north(vbar_c * v_c) - vbar_c * v_c) / dy
        ubar = 0.5 * (u + north(u))
        fx = ubar * face_value(v, ubar, -1, m3v, lim)
        bx = (fx - west(fx)) / dx
        wbv = 0.5 * (w + north(w))
        fzv = zpad(wbv[1:nz] * face_value_z(v, wbv, m3v, lim), nz)
        bz = (fzv[:nz] - fzv[1:nz + 1]) / dz
        return ax + ay + az, bx + by + bz
    ubar_c = 0.5 * (west(u) + u)
    ax = (east(ubar_c) ** 2 - ubar_c ** 2) / dx
    vbar = 0.5 * (v + east(v))
    fy = vbar * (0.5 * (u + north(u)))
    ay = (fy - south(fy)) / dy
    wbar = 0.5 * (w + east(w))
    fz = zpad(wbar[1:nz] * 0.5 * (u[:-1] + u[1:]), nz)
    az = (fz[:nz] - fz[1:nz + 1]) / dz
    vbar_c = 0.5 * (south(v) + v)
    by = (north(vbar_c) ** 2 - vbar_c ** 2) / dy
    ubar = 0.5 * (u + north(u))
    fx = ubar * (0.5 * (v + east(v)))
    bx = (fx - west(fx)) / dx
    wbv = 0.5 * (w + north(w))
    fzv = zpad(wbv[1:nz] * 0.5 * (v[:-1] + v[1:]), nz)
    bz = (fzv[:nz] - fzv[1:nz + 1]) / dz
    return ax + ay + az, bx + by + bz


def rho_teos10(CT, SA, z):
    """The oracle's polyTEOS10-bsq Horner form (oracle.rho_teos10) on tensors."""
    c = orc._C
    r00, r01, r02, r03, r04, r05 = orc._R0
    zh = z * orc.R1_Z0
    ss = torch.sqrt((SA + orc.RDELTA_S) * orc.R1_S0)
    tt = CT * orc.R1_T0
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


def rho_anomaly(p, T, S, z):
    if p.eos == "linear":
        return p.rho0 * (-p.alpha_t * (T - p.t0) + p.beta_s * (S - p.s0))
    if p.eos == "seos":
        a0, b0, lam1, lam2, mu1, mu2, nu_ts = orc._SEOS
        Ta, Sa = T - 10.0, S - 35.0
        return (-a0 * (1.0 + 0.5 * lam1 * Ta + mu1 * z) * Ta + b0 * (1.0 - 0.5 * lam2 * Sa - mu2 * z) * Sa
                - nu_ts * Ta * Sa)
    return rho_teos10(T, S, z) - p.rho0


class HelmSolve(torch.autograd.Function):
    """x = A^-1 b on the wet cells by PCG-Jacobi to rtol 1e-15; A is symmetric
    there, so the backward is the same solve."""

    @staticmethod
    def _pcg(op, b):
        b = b * op["mask"]
        x = torch.zeros_like(b)
        nb = torch.linalg.vector_norm(b)
        if float(nb) == 0.0:
            return x
        r = b.clone()
        z = op["inv_diag"] * r
        p = z.clone()
        rz = torch.sum(r * z)
        for _ in range(20000):
            Ap = op["apply"](p)
            alpha = rz / torch.sum(p * Ap)
            x = x + alpha * p
            r = r - alpha * Ap
            if float(torch.linalg.vector_norm(r)) <= 1e-15 * float(nb):
                break
            z = op["inv_diag"] * r
            rz_new = torch.sum(r * z)
            p = z + (rz_new / rz) * p
            rz = rz_new
        return x

    @staticmethod
    def forward(ctx, b, op):
        ctx.op = op
        return HelmSolve._pcg(op, b.detach())

    @staticmethod
    def backward(ctx, g):
        return HelmSolve._pcg(ctx.op, g), None


class TorchStep:
    """One step of the theta scheme (closure none, TS tracers) in float64 torch.

    ``p`` is an OceanParams; ``H``, ``mask``, ``dzr`` the domain as for the
    oracle. ``step(state, taux_c)`` takes a dict of tensors (eta, u, v, b, T, S)
    and the surface x-stress at centres; every output is differentiable with
    respect to every input, the stress included."""

    def __init__(self, p, H, mask, dzr=None, device="cuda"):
        if p.scheme_name != "theta" or p.closure != "none" or p.tracers != "TS":
            raise ValueError("the torch restatement covers theta, closure none, TS tracers")
        self.p, self.dev = p, device
        g = orc.Geometry(p, H, mask, dzr)
        self.geo = g
        T = lambda a: _t(a, device)  # noqa: E731
        self.dz3, self.m3 = T(g.dz3), T(g.mask3)
        self.m3u, self.m3v = T(g.mask3u), T(g.mask3v)
        self.dz3u, self.dz3v = T(g.dz3u), T(g.dz3v)
        self.zc = T(g.zc)
        self.mask, self.mask_u, self.mask_v = T(g.mask), T(g.mask_u), T(g.mask_v)
        self.dx, self.dy, self.dt = g.dx, g.dy, float(p.dt)
        nz, ny, nx = g.nz, g.ny, g.nx
        Km = orc.np.full((nz + 1, ny, nx), p.nu)
        Kh = orc.np.full((nz + 1, ny, nx), p.kappa)
        self.Km, self.Kh = T(Km), T(Kh)
        tri_m = orc.implicit_coeffs(Km, g.dz3, self.dt, p.theta_v, p.bottom_drag, g.mask3)
        tri_b = orc.implicit_coeffs(Kh, g.dz3, self.dt, p.theta_v, 0.0, g.mask3)
        q = orc.thomas(*tri_m, orc.np.ones((nz, ny, nx)))
        self.tri_m = tuple(T(a) for a in tri_m)
        self.tri_b = tuple(T(a) for a in tri_b)
        self.q = T(q)
        Ku = orc.np.sum(g.dz3u * orc.np.minimum(q, orc._east(q)), axis=0) * g.mask_u
        Kv = orc.np.sum(g.dz3v * orc.np.minimum(q, orc._north(q)), axis=0) * g.mask_v
        op = orc.HelmOp(nx, ny, p.lx, p.ly, p.g * p.theta ** 2 * self.dt ** 2, Ku, Kv, g.mask)
        Kut, Kvt, mt = T(Ku), T(Kv), T(g.mask)
        coef, dx2, dy2 = op.coef, op.dx ** 2, op.dy ** 2

        def apply(x):
            x = x * mt
            fx = Kut * (east(x) - x)
            fy = Kvt * (north(x) - x)
            lap = (fx - west(fx)) / dx2 + (fy - south(fy)) / dy2
            return (x - coef * lap) * mt + x * (1.0 - mt)

        self.helm = {"apply": apply, "inv_diag": T(op.inv_diag), "mask": mt}
        self.dz_nom = p.h0 / nz
        self.bottom = T(orc._bottom_cells(g.mask3).astype(float))
        self.inv_dz3 = T(orc.inv_pos(g.dz3))
        self.inv_dz3u = T(orc.inv_pos(g.dz3u))
        self.inv_dz3v = T(orc.inv_pos(g.dz3v))

    # -- pieces (oracle functions of the same names)
    def centre_spacing(self, dz3):
        return torch.cat([dz3[:1], 0.5 * (dz3[:-1] + dz3[1:]), dz3[-1:]], 0)

    def explicit_diffusion(self, f, K, dz3, inv_dz3, surf, drag):
        nz = f.shape[0]
        dzi = self.centre_spacing(dz3)
        inv_dzi = torch.where(dzi > 0, 1.0 / torch.where(dzi > 0, dzi, torch.ones_like(dzi)),
                              torch.zeros_like(dzi))
        inner = K[1:nz] * (f[:nz - 1] - f[1:nz]) * inv_dzi[1:nz]
        inner = torch.where(self.bottom[:nz - 1] > 0, torch.zeros_like(inner), inner)
        flux = torch.cat([surf[None], inner, torch.zeros_like(f[:1])], 0)
        dragc = drag * f * self.bottom
        out = (flux[:nz] - flux[1:nz + 1]) * inv_dz3
        return (out - dragc * inv_dz3) * (self.m3 > 0)

    def w_from(self, u, v):
        td = self.m3 * ((self.dz3u * u - west(self.dz3u * u)) / self.dx
                        + (self.dz3v * v - south(self.dz3v * v)) / self.dy)
        w = -torch.flip(torch.cumsum(torch.flip(td, [0]), 0), [0])
        return torch.cat([w, torch.zeros_like(w[:1])], 0)

    def pgf(self, b):
        dz3, zc = self.dz3, self.zc
        above = torch.cat([torch.zeros_like(b[:1]), torch.cumsum((dz3 * b)[:-1], 0)], 0)
        phi = 0.5 * dz3 * b + above
        p = self.p
        if p.pgf == "remove":
            total = torch.sum(dz3, 0, keepdim=True)
            inv = torch.where(total > 0, 1.0 / torch.where(total > 0, total, torch.ones_like(total)),
                              torch.zeros_like(total))
            phi = phi - torch.sum(dz3 * phi, 0, keepdim=True) * inv
        if not p.pgf_correction:
            return (self.m3u * (east(phi) - phi) / self.dx * self.m3u,
                    self.m3v * (north(phi) - phi) / self.dy * self.m3v)
        out = []
        for axis, fm, delta in ((-1, self.m3u, self.dx), (-2, self.m3v, self.dy)):
            phi_r, b_r, z_r = shift(phi, axis, -1), shift(b, axis, -1), shift(zc, axis, -1)
            zf = 0.5 * (zc + z_r)
            out.append(fm * ((phi_r + b_r * (zf - z_r)) - (phi + b * (zf - zc))) / delta)
        return out[0], out[1]

    def v_at_u(self, v, mv, mu):
        vs, ms = south(v), south(mv)
        pairs = [(v, mv), (vs, ms), (east(v), east(mv)), (east(vs), east(ms))]
        num = sum(w * f for f, w in pairs)
        den = sum(w for _, w in pairs)
        return torch.where(den > 0, num / torch.where(den > 0, den, torch.ones_like(den)),
                           torch.zeros_like(den)) * mu

    def u_at_v(self, u, mu, mv):
        uw, mw = west(u), west(mu)
        pairs = [(u, mu), (uw, mw), (north(u), north(mu)), (north(uw), north(mw))]
        num = sum(w * f for f, w in pairs)
        den = sum(w for _, w in pairs)
        return torch.where(den > 0, num / torch.where(den > 0, den, torch.ones_like(den)),
                           torch.zeros_like(den)) * mv

    def hlap(self, f, m):
        gx = self.m3u * (east(f) - f) / self.dx
        gy = self.m3v * (north(f) - f) / self.dy
        return m * ((gx - west(gx)) / self.dx + (gy - south(gy)) / self.dy)

    def div2(self, U, V):
        return self.mask * ((U - west(U)) / self.dx + (V - south(V)) / self.dy)

    def tracer_adv(self, c, u, v, w):
        p = self.p
        s = p.advection
        if s == "centered2":
            cx, cy = 0.5 * (c + east(c)), 0.5 * (c + north(c))
        elif s in ("up3", "up3_tvd"):
            cx = face_value(c, u, -1, self.m3, s == "up3_tvd")
            cy = face_value(c, v, -2, self.m3, s == "up3_tvd")
        else:
            cx = torch.where(u > 0, c, east(c))
            cy = torch.where(v > 0, c, north(c))
        fx = self.dz3u * u * cx
        fy = self.dz3v * v * cy
        inv = self.inv_dz3
        hdiv = ((fx - west(fx)) / self.dx + (fy - south(fy)) / self.dy) * inv
        nz = c.shape[0]
        if s in ("up3", "up3_tvd"):
            inner = face_value_z(c, w, self.m3, s == "up3_tvd")
        else:
            inner = 0.5 * (c[:nz - 1] + c[1:nz])
        cf = torch.cat([c[:1], inner, torch.zeros_like(c[:1])], 0)
        vdiv = (w[:nz] * cf[:nz] - w[1:] * cf[1:]) * inv
        return (hdiv + vdiv) * self.m3

    def tracer(self, c, u, v, w, surf):
        p, dt = self.p, self.dt
        tend = torch.zeros_like(c)
        if p.advection != "none":
            tend = tend - self.tracer_adv(c, u, v, w)
        if p.k_h > 0.0:
            tend = tend + p.k_h * self.hlap(c, self.m3)
        rhs = c + dt * tend + (1.0 - p.theta_v) * dt * self.explicit_diffusion(c, self.Kh, self.dz3, self.inv_dz3,
                                                                             surf, 0.0)
        top = rhs[0] + p.theta_v * dt * surf * self.inv_dz3[0]
        rhs = torch.cat([top[None], rhs[1:]], 0)
        return thomas(*self.tri_b, rhs) * self.m3

    def buoyancy(self, T, S):
        p = self.p
        return -p.g * rho_anomaly(p, T, S, self.zc) / p.rho0 * self.m3

    def stress(self, taux_c, tauy_c=None):
        p = self.p
        ty = torch.zeros_like(taux_c) if tauy_c is None else tauy_c
        tau_u = (0.5 * (taux_c + east(taux_c))) / p.rho0 * self.m3u[0]
        tau_v = (0.5 * (ty + north(ty))) / p.rho0 * self.m3v[0]
        return tau_u, tau_v

    def step(self, s: dict, taux_c, tauy_c=None) -> dict:
        p, dt = self.p, self.dt
        th, tc, thv = p.theta, p.theta_cor, p.theta_v
        m3 = self.m3
        tau_u, tau_v = self.stress(taux_c, tauy_c)
        u, v, b, eta, Tt, Ss = s["u"], s["v"], s["b"], s["eta"], s["T"], s["S"]
        pgx, pgy = self.pgf(b)
        avp_v = self.v_at_u(v, self.m3v, self.m3u)
        avp_u = self.u_at_v(u, self.m3u, self.m3v)
        dzu = self.explicit_diffusion(u, self.Km, self.dz3u, self.inv_dz3u, tau_u, p.bottom_drag)
        dzv = self.explicit_diffusion(v, self.Km, self.dz3v, self.inv_dz3v, tau_v, p.bottom_drag)
        w_old = self.w_from(u, v)
        ex_u = torch.zeros_like(u)
        ex_v = torch.zeros_like(v)
        if p.advection != "none":
            au, av = momentum_adv(u, v, w_old, self.dx, self.dy, self.dz_nom, self.m3u, self.m3v, p.advection)
            ex_u = ex_u - au * self.m3u
            ex_v = ex_v - av * self.m3v
        if p.a_h > 0.0:
            ex_u = ex_u + p.a_h * self.hlap(u, self.m3u)
            ex_v = ex_v + p.a_h * self.hlap(v, self.m3v)
        st_u = torch.cat([(thv * dt * tau_u * self.inv_dz3u[0])[None], torch.zeros_like(u[1:])], 0) + dt * ex_u
        st_v = torch.cat([(thv * dt * tau_v * self.inv_dz3v[0])[None], torch.zeros_like(v[1:])], 0) + dt * ex_v
        gx_eta = (self.mask_u * (east(eta) - eta) / self.dx)[None] * self.m3u
        gy_eta = (self.mask_v * (north(eta) - eta) / self.dy)[None] * self.m3v
        div_old = self.div2(torch.sum(self.dz3u * u, 0), torch.sum(self.dz3v * v, 0))
        u_it, v_it, eta_new = u, v, eta
        for _ in range(p.n_picard):
            v_cor = (1.0 - tc) * avp_v + tc * self.v_at_u(v_it, self.m3v, self.m3u)
            u_cor = (1.0 - tc) * avp_u + tc * self.u_at_v(u_it, self.m3u, self.m3v)
            gu = u + dt * (p.f0 * v_cor + pgx) - p.g * dt * (1.0 - th) * gx_eta + (1.0 - thv) * dt * dzu
            gv = v + dt * (-p.f0 * u_cor + pgy) - p.g * dt * (1.0 - th) * gy_eta + (1.0 - thv) * dt * dzv
            gh_u = thomas(*self.tri_m, gu + st_u) * m3
            gh_v = thomas(*self.tri_m, gv + st_v) * m3
            div_g = self.div2(torch.sum(self.dz3u * gh_u, 0), torch.sum(self.dz3v * gh_v, 0))
            rhs = eta - dt * ((1.0 - th) * div_old + th * div_g)
            eta_new = HelmSolve.apply(rhs, self.helm)
            gxn = (self.mask_u * (east(eta_new) - eta_new) / self.dx)[None] * self.m3u
            gyn = (self.mask_v * (north(eta_new) - eta_new) / self.dy)[None] * self.m3v
            u_it = (gh_u - p.g * dt * th * self.q * gxn) * m3
            v_it = (gh_v - p.g * dt * th * self.q * gyn) * m3
        w = self.w_from(u_it, v_it)
        fT = torch.full_like(eta, p.q_heat / (p.rho0 * p.cp))
        fS = torch.full_like(eta, p.q_salt)
        T_new = self.tracer(Tt, u_it, v_it, w, fT)
        S_new = self.tracer(Ss, u_it, v_it, w, fS)
        return {"u": u_it, "v": v_it, "b": self.buoyancy(T_new, S_new), "eta": eta_new, "T": T_new, "S": S_new}
