"""FP64 autograd reference of the SPMHD step -- test infrastructure only.

A PyTorch restatement (CPU, float64, dense all-pairs, small cases only) of
the reference's literal PEC step with the single density pass --
``MHDStep`` (src/integrator.py:12-82), the ten groups of
``MHDScheme.get_equations`` (src/scheme.py:66-81; src/equations.py) -- and
of the warm-up (src/application.py:110-132), traced by torch.autograd.  It
is the independent check of the library's derivative forms: their gradient
must equal the one autograd takes through this code.  Only tests import it.

Non-differentiable points follow the library's convention: sqrt and |.| have
derivative 0 at 0, and max/min send the derivative to the selected
argument only.
"""

from __future__ import annotations

import math

import torch

KERNEL_R = {"cubic": 2.0, "quintic": 3.0, "wendland_c2": 2.0, "wendland_c4": 2.0, "wendland_c6": 2.0}
_TINY = 1e-300


def _norm(kernel, dim):
    table = {"cubic": {2: 10.0 / (7.0 * math.pi), 3: 1.0 / math.pi},
             "quintic": {2: 7.0 / (478.0 * math.pi), 3: 1.0 / (120.0 * math.pi)},
             "wendland_c2": {2: 7.0 / (4.0 * math.pi), 3: 21.0 / (16.0 * math.pi)},
             "wendland_c4": {2: 9.0 / (4.0 * math.pi), 3: 495.0 / (256.0 * math.pi)},
             "wendland_c6": {2: 78.0 / (28.0 * math.pi), 3: 1365.0 / (512.0 * math.pi)}}
    return table[kernel][dim]


def ssqrt(x):
    """sqrt with derivative 0 at 0."""
    pos = x > 0
    return torch.where(pos, torch.sqrt(torch.where(pos, x, torch.ones_like(x))), torch.zeros_like(x))


def pmax(a, b):
    return torch.where(b > a, b, a)


def pmin(a, b):
    return torch.where(b < a, b, a)


def w_dw(kernel, q, dim):
    """Unnormalised w(q), dw/dq (pysph kernels, restated)."""
    z = torch.zeros_like(q)
    if kernel == "cubic":
        t = 2.0 - q
        w = torch.where(q > 2, z, torch.where(q > 1, 0.25 * t * t * t, 1.0 - 1.5 * q * q * (1.0 - 0.5 * q)))
        dw = torch.where(q > 2, z, torch.where(q > 1, -0.75 * t * t, -3.0 * q * (1.0 - 0.75 * q)))
        return w, dw
    if kernel == "quintic":
        t3, t2, t1 = 3.0 - q, 2.0 - q, 1.0 - q
        w = t3 ** 5 - torch.where(q <= 2, 6.0 * t2 ** 5, z) + torch.where(q <= 1, 15.0 * t1 ** 5, z)
        dw = -5.0 * t3 ** 4 + torch.where(q <= 2, 30.0 * t2 ** 4, z) - torch.where(q <= 1, 75.0 * t1 ** 4, z)
        return torch.where(q > 3, z, w), torch.where(q > 3, z, dw)
    s = 1.0 - 0.5 * q
    if kernel == "wendland_c2":
        w, dw = s ** 4 * (2.0 * q + 1.0), -5.0 * q * s ** 3
    elif kernel == "wendland_c4":
        w, dw = s ** 6 * (35.0 / 12.0 * q * q + 3.0 * q + 1.0), -14.0 / 3.0 * q * (1.0 + 2.5 * q) * s ** 5
    else:
        w = s ** 8 * (4.0 * q ** 3 + 6.25 * q * q + 4.0 * q + 1.0)
        dw = -5.5 * q * (1.0 + 3.5 * q + 4.0 * q * q) * s ** 7
    return torch.where(q >= 2, z, w), torch.where(q >= 2, z, dw)


class Step:
    """prm: the library's flat parameter dict (single density pass)."""

    def __init__(self, prm):
        self.p = prm
        self.dim = prm["dim"]
        self.R = KERNEL_R[prm["kernel"]]
        self.norm = _norm(prm["kernel"], self.dim)
        self.L = [prm["hi"][a] - prm["lo"][a] for a in range(3)]

    # --- geometry
    def pairs(self, x, h):
        """x_ij (3, n, n) minimum image on the values, r_ij, neighbour mask."""
        xs = []
        for a in range(3):
            if a >= self.dim:
                xs.append(torch.zeros_like(x[0])[:, None] * torch.zeros_like(x[0])[None, :])
                continue
            d = x[a][:, None] - x[a][None, :]
            if self.p["periodic"][a]:
                L = self.L[a]
                shift = torch.where(d.detach() > 0.5 * L, -L, 0.0) * 1.0
                d = d + shift
                shift2 = torch.where(d.detach() < -0.5 * L, L, 0.0) * 1.0
                d = d + shift2
            xs.append(d)
        xij = torch.stack(xs)
        r2 = (xij[0] * xij[0] + xij[1] * xij[1]) + xij[2] * xij[2]
        rh = (self.R * h) ** 2
        mask = (r2.detach() < rh.detach()[:, None]) | (r2.detach() < rh.detach()[None, :])
        return xij, ssqrt(r2), mask

    def hfac(self, h1):
        return self.norm * h1 ** self.dim

    def kernel(self, r, h):
        """W(r, h), dW/dr factor (grad W = g * x_ij), dW/dh for h per row."""
        h1 = 1.0 / h
        q = r * h1
        w, dw = w_dw(self.p["kernel"], q, self.dim)
        fac = self.hfac(h1)
        W = w * fac
        big = r > 1e-12
        g = torch.where(big, fac * dw * h1 / torch.where(big, r, torch.ones_like(r)), torch.zeros_like(r))
        dWdh = -(fac * h1 * (dw * q + w * float(self.dim)))
        return W, g, dWdh

    # --- groups
    def rhs(self, s, amax, converged):
        p, dim = self.p, self.dim
        m = s["m"]
        mu0 = p["mu0"]
        # G1 single density pass (converged particles keep h and Omega)
        xij, r, mask = self.pairs(s["x"], s["h"])
        W, g, dWdh = self.kernel(r, s["h"][:, None])
        rho_sum = torch.sum(torch.where(mask, m[None, :] * W, 0.0), 1)
        dwdh = torch.sum(torch.where(mask, m[None, :] * dWdh, 0.0), 1)
        hk = s["h"] / p["hfact"]
        rhoi = m / hk ** dim
        dhdrho = -s["h"] / (dim * rhoi)
        omega_new = 1.0 / (1.0 - dhdrho * dwdh)
        h_new = p["hfact"] * (m / rho_sum) ** (1.0 / dim)
        if converged:
            h_new, omega = s["h"], s["omega"]
        else:
            omega = omega_new
        # G2, G3, G5
        hk = h_new / p["hfact"]
        rho = m / hk ** dim
        pres = (p["gamma"] - 1.0) * rho * s["epred"]
        cs = ssqrt(p["gamma"] * pres / rho)
        b = [s["bpred"][a] * rho for a in range(3)]
        # pairs with the new h
        xij, r, mask = self.pairs(s["x"], h_new)
        _, gi, _ = self.kernel(r, h_new[:, None])
        _, gj, _ = self.kernel(r, h_new[None, :])
        dwi = [gi * xij[a] for a in range(3)]
        dwj = [gj * xij[a] for a in range(3)]
        M = torch.where(mask, 1.0, 0.0)
        mj = m[None, :]
        v = s["vpred"]
        dv = [v[a][:, None] - v[a][None, :] for a in range(3)]
        # G4 Cullen-Dehnen (src/equations.py:318-429)
        run = [mj * dwi[b_] for b_ in range(3)]
        rr = [torch.sum(M * (-xij[ia] * run[ib]), 1) for ia, ib in ((0, 0), (0, 1), (0, 2), (1, 1), (1, 2), (2, 2))]
        acc = s["a"]
        da = [acc[a][:, None] - acc[a][None, :] for a in range(3)]
        vv = [torch.sum(M * dv[a] * run[bb], 1) for a in range(3) for bb in range(3)]
        aa = [torch.sum(M * da[a] * run[bb], 1) for a in range(3) for bb in range(3)]
        rxx, rxy, rxz, ryy, ryz, rzz = rr
        denom = rxx * ryy * rzz + 2.0 * rxy * rxz * ryz - rxx * ryz * ryz - ryy * rxz * rxz - rzz * rxy * rxy
        termnorm = omega / rho
        if dim == 3:
            inv = torch.abs(denom.detach()) > 2.2250738585072014e-308
            dd = 1.0 / torch.where(inv, denom, torch.ones_like(denom))
            txx, txy, txz = ryy * rzz - ryz * ryz, rxz * ryz - rzz * rxy, rxy * ryz - rxz * ryy
            tyy, tyz, tzz = rzz * rxx - rxz * rxz, rxy * rxz - rxx * ryz, rxx * ryy - rxy * rxy
            gax = (aa[0] * txx + aa[1] * txy + aa[2] * txz) * dd
            gay = (aa[3] * txy + aa[4] * tyy + aa[5] * tyz) * dd
            gaz = (aa[6] * txz + aa[7] * tyz + aa[8] * tzz) * dd
            div_a = torch.where(inv, -(gax + gay + gaz), -termnorm * (aa[0] + aa[4] + aa[8]))
            G = []
            for a in range(3):
                row = (vv[3 * a], vv[3 * a + 1], vv[3 * a + 2])
                G += [torch.where(inv, -((row[0] * txx + row[1] * txy + row[2] * txz) * dd), -termnorm * row[0]),
                      torch.where(inv, -((row[0] * txy + row[1] * tyy + row[2] * tyz) * dd), -termnorm * row[1]),
                      torch.where(inv, -((row[0] * txz + row[1] * tyz + row[2] * tzz) * dd), -termnorm * row[2])]
        else:
            div_a = -termnorm * (aa[0] + aa[4] + aa[8])
            G = [-termnorm * vv[k] for k in range(9)]
        divvdt = div_a - (G[0] * G[0] + G[4] * G[4] + G[8] * G[8] + 2.0 * (G[1] * G[3] + G[2] * G[6] + G[5] * G[7]))
        divv = G[0] + G[4] + G[8]
        curl = [G[7] - G[5], G[2] - G[6], G[3] - G[1]]
        comp = pmax(-divv, torch.zeros_like(divv))
        fac = comp * comp
        den = fac + curl[0] ** 2 + curl[1] ** 2 + curl[2] ** 2
        xi = torch.where(den > 0, fac / torch.where(den > 0, den, torch.ones_like(den)), torch.ones_like(den))
        source = 10.0 * h_new * h_new * xi * pmax(-divvdt, torch.zeros_like(divvdt))
        aloc = pmax(pmin(source / (cs * cs), amax * torch.ones_like(source)), p["alpha_min"] * torch.ones_like(source))
        # G6 MHDAccelerations
        rho_i, rho_j = rho[:, None], rho[None, :]
        p_i, p_j = pres[:, None], pres[None, :]
        om_i, om_j = omega[:, None], omega[None, :]
        bi2 = b[0] ** 2 + b[1] ** 2 + b[2] ** 2
        vwave = ssqrt(cs * cs + bi2 / (mu0 * rho))
        vw_i, vw_j = vwave[:, None], vwave[None, :]
        small = r < 1e-8
        rs = torch.where(small, torch.ones_like(r), r)
        runi = [torch.where(small, torch.zeros_like(r), xij[a] / rs) for a in range(3)]
        dot = dv[0] * runi[0] + dv[1] * runi[1] + dv[2] * runi[2]
        grad_i = om_i * (runi[0] * dwi[0] + runi[1] * dwi[1] + runi[2] * dwi[2])
        grad_j = om_j * (runi[0] * dwj[0] + runi[1] * dwj[1] + runi[2] * dwj[2])
        div = torch.sum(M * mj * dot * grad_i, 1)
        vsig2 = ssqrt(torch.abs(p_i - p_j) / (0.5 * (rho_i + rho_j)))
        alpha = s["alpha1"]
        vav_i = pmax(alpha[:, None] * vw_i - 2.0 * dot, torch.zeros_like(dot))
        vav_j = pmax(alpha[None, :] * vw_j - 2.0 * dot, torch.zeros_like(dot))
        av = torch.where(dot < 0, torch.ones_like(dot), torch.zeros_like(dot))
        q_i = -0.5 / rho_i * vav_i * dot * p["av"] * av
        q_j = -0.5 / rho_j * vav_j * dot * p["av"] * av
        pir, pjr = p_i / rho_i ** 2, p_j / rho_j ** 2
        a6 = [torch.sum(M * (-mj * (q_i * om_i * dwi[a] + q_j * om_j * dwj[a]) - mj * (pir * om_i * dwi[a] +
                                                                                        pjr * om_j * dwj[a])), 1)
              for a in range(3)]
        e = s["epred"]
        ae6 = torch.sum(M * (mj * q_i * dot * grad_i + mj * pir * om_i * (dv[0] * dwi[0] + dv[1] * dwi[1] +
                                                                           dv[2] * dwi[2]) +
                             p["ac"] * vsig2 * (e[:, None] - e[None, :]) * (0.5 * mj / rho_i * grad_i +
                                                                             0.5 * mj / rho_j * grad_j)), 1)
        # G8 / G9 unit vector
        big = r > 1e-12
        rb = torch.where(big, r, torch.ones_like(r))
        run2 = [torch.where(big, xij[a] / rb, torch.zeros_like(r)) for a in range(3)]
        g2i = om_i * (run2[0] * dwi[0] + run2[1] * dwi[1] + run2[2] * dwi[2])
        g2j = om_j * (run2[0] * dwj[0] + run2[1] * dwj[1] + run2[2] * dwj[2])
        brho = [b[a] / rho for a in range(3)]
        bro2 = (brho[0] ** 2 + brho[1] ** 2 + brho[2] ** 2) / mu0
        gradp = mj * (0.5 * bro2[:, None] * g2i + 0.5 * bro2[None, :] * g2j)
        a8 = []
        for a in range(3):
            pi = sum((-mj * brho[a][:, None] * brho[c][:, None] / mu0) * run2[c] for c in range(3))
            pj = sum((-mj * brho[a][None, :] * brho[c][None, :] / mu0) * run2[c] for c in range(3))
            a8.append(torch.sum(M * (-run2[a] * gradp - (pi * g2i + pj * g2j)), 1))
        bi = [b[a][:, None] for a in range(3)]
        bj = [b[a][None, :] for a in range(3)]
        proj_bi = sum(bi[a] * run2[a] for a in range(3))
        proj_bj = sum(bj[a] * run2[a] for a in range(3))
        db = [bi[a] - bj[a] for a in range(3)]
        proj_db = sum(db[a] * run2[a] for a in range(3))
        delta_b2 = db[0] ** 2 + db[1] ** 2 + db[2] ** 2
        pgi, pgj = mj / rho_i ** 2 * g2i, mj / rho_j ** 2 * g2j
        projv = sum(dv[a] * run2[a] for a in range(3))
        dvt = [dv[a] - projv * run2[a] for a in range(3)]
        vsig_b = ssqrt(dvt[0] ** 2 + dvt[1] ** 2 + dvt[2] ** 2)
        d_diss = 0.5 * (pgi + pgj) * vsig_b * p["ar"]
        psi = s["psipred"]
        dpsi = pgi * psi[:, None] * (p["clean_speed"] * vw_i) + pgj * psi[None, :] * (p["clean_speed"] * vw_j)
        ab = [torch.sum(M * (-(pgi * proj_bi) * dv[a] + d_diss * db[a] - dpsi * run2[a]), 1) for a in range(3)]
        ae9 = torch.sum(M * (-0.5 * delta_b2 * d_diss / mu0), 1)
        divbs = torch.sum(M * (pgi * proj_bi + pgj * proj_bj), 1)
        divbd = torch.sum(M * (-mj * proj_db * g2i), 1)
        # posts (G6 post, G7, G9 post, G10 with the limiter inactive)
        divv_f = -div / rho
        ah = h_new * divv_f / dim
        ch = p["clean_speed"] * vwave
        apsi = -ch * divbd / rho - p["clean_damp"] * psi * ch / h_new - 0.5 * (1.0 if p["clean_speed"] > 0 else 0.0) * \
            psi * divv_f
        ae = ae6 + ae9
        pbeta = 2.0 * mu0 * pres / bi2
        frac = pmax(torch.zeros_like(pbeta), pmin(torch.ones_like(pbeta), (10.0 - pbeta) * 0.125))
        frac = torch.where(bi2 > 0, frac, torch.zeros_like(frac))
        au = [(a6[a] + a8[a]) + (-b[a] * divbs * frac / mu0) for a in range(3)]
        return dict(h=h_new, omega=omega, rho=rho, cs=cs, b=b, aloc=aloc, a=au, ae=ae, ah=ah, ab=ab, apsi=apsi)

    # --- integrator
    def run(self, ic, amax, dts):
        """Warm-up, then the PEC steps with sizes dts; returns the final
        magnetic energy sum m |B|^2 / (2 mu0 rho)."""
        p, dim = self.p, self.dim
        m = ic["m"]
        x = [ic["x"], ic["y"], ic["z"]]
        v = [ic["u"], ic["v"], ic["w"]]
        b_ic = [ic["Bx"], ic["By"], ic["Bz"]]
        rho, h, e = ic["rho"], ic["h"], ic["e"]
        zero = torch.zeros_like(m)
        a, ae, ah, ab, apsi = [zero] * 3, zero, zero, [zero] * 3, zero
        alpha1, aloc, cs, omega = ic["alpha1"], zero, zero, zero + 1.0

        def rhs(bev, psi, converged, state_omega):
            return self.rhs(dict(x=x, h=h, m=m, epred=e, bpred=bev, vpred=v, a=a, alpha1=alpha1, psipred=psi,
                                 omega=state_omega), amax, converged)

        # warm-up (src/application.py:110-132)
        bev = [b_ic[c] / rho for c in range(3)]
        o = rhs(bev, zero, False, omega)
        h, omega, rho, cs, aloc, a, ae, ah, ab, apsi = (o["h"], o["omega"], o["rho"], o["cs"], o["aloc"], o["a"],
                                                        o["ae"], o["ah"], o["ab"], o["apsi"])
        bev = [b_ic[c] / rho for c in range(3)]
        for _ in range(2):
            o = rhs(bev, zero, True, omega)
            h, rho, cs, aloc, a, ae, ah, ab, apsi = (o["h"], o["rho"], o["cs"], o["aloc"], o["a"], o["ae"], o["ah"],
                                                     o["ab"], o["apsi"])
        psi = zero
        for dt in dts:
            dtb2 = 0.5 * dt
            vh = [v[c] + dtb2 * a[c] for c in range(3)]
            vp = [v[c] + dt * a[c] for c in range(3)]
            xn = list(x)
            for c in range(dim):
                xc = x[c] + dt * vh[c]
                if p["periodic"][c]:
                    lo, hi, L = p["lo"][c], p["hi"][c], self.L[c]
                    xc = xc + torch.where(xc.detach() < lo, L, 0.0)
                    xc = xc - torch.where(xc.detach() > hi, L, 0.0)
                xn[c] = xc
            eh, ep = e + dtb2 * ae, e + dt * ae
            hp = h + dt * ah
            decay = 0.1 * cs / hp
            alpha1 = torch.where(alpha1 < aloc, aloc, (alpha1 + dt * aloc * decay) / (1.0 + dt * decay))
            bh = [bev[c] + dtb2 * ab[c] for c in range(3)]
            bp = [bev[c] + dt * ab[c] for c in range(3)]
            psih, psip = psi + dtb2 * apsi, psi + dt * apsi
            x, h = xn, hp
            o = self.rhs(dict(x=x, h=h, m=m, epred=ep, bpred=bp, vpred=vp, a=a, alpha1=alpha1, psipred=psip,
                              omega=omega), amax, False)
            h, omega, rho, cs, aloc, a, ae, ah, ab, apsi = (o["h"], o["omega"], o["rho"], o["cs"], o["aloc"],
                                                            o["a"], o["ae"], o["ah"], o["ab"], o["apsi"])
            v = [vh[c] + dtb2 * a[c] for c in range(3)]
            e = eh + dtb2 * ae
            bev = [bh[c] + dtb2 * ab[c] for c in range(3)]
            psi = psih + dtb2 * apsi
        bsq = sum((bev[c] * rho) ** 2 for c in range(3))
        return torch.sum(m * bsq / (2.0 * p["mu0"] * rho))
