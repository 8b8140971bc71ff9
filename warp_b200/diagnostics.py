"""Beam moments of getzmmnt (pywarp90/top.F:521-1700): the global moments
(pnum, xbar, ..., epsx, ...) and the moments on a z grid (pnumz, xbarz, ...,
epsxz, ...) from the 33 moment sums that wg_zmoments accumulates on the GPU.

finalize() is itask = 3 of getzmmnt (top.F:1317-1700): divide the sums by
the particle number, subtract the products of the averages, and form the rms
sizes and the emittances. It runs on the host with numpy over the small
arrays of sums, elementwise in the reference's operation order; the same
code turns the oracle's sums into moments in the tests.

The sums are indexed 0..32 for the reference's moments 1..33:
  0 pnum, 1 x, 2 y, 3 z, 4 x', 5 y', 6 vx, 7 vy, 8 vz, 9 xy, 10 x'y', 11 x^2,
  12 y^2, 13 z^2, 14 x'^2, 15 y'^2, 16 vx^2, 17 vy^2, 18 vz^2, 19 xx', 20 yy',
  21 z vz, 22 xy', 23 yx', 24 x vz, 25 y vz, 26 vx vz, 27 vy vz, 28 x vx,
  29 y vy, 30 x vy, 31 y vx, 32 vx vy.
"""
import numpy as np

from .constants import clight

SMALLPOS = 1.0e-36

_BARS = ("xbar", "ybar", "zbar", "xpbar", "ypbar", "vxbar", "vybar", "vzbar", "xybar", "xpypbar", "xsqbar",
         "ysqbar", "zsqbar", "xpsqbar", "ypsqbar", "vxsqbar", "vysqbar", "vzsqbar", "xxpbar", "yypbar", "zvzbar",
         "xypbar", "yxpbar", "xvzbar", "yvzbar", "vxvzbar", "vyvzbar", "xvxbar", "yvybar", "xvybar", "yvxbar",
         "vxvybar")


def finalize(sums, suffix=""):
    """Moments from sums of shape (33,) or (nz+1, 33); returns a dict whose
    keys carry `suffix` ("z" for the z-grid arrays, as pnumz, xrmsz, ...)."""
    s = np.asarray(sums, dtype=np.float64)
    pnumi = 1. / (s[..., 0] + SMALLPOS)
    m = {"pnum": s[..., 0].copy()}
    for k, name in enumerate(_BARS):
        m[name] = s[..., k + 1] * pnumi
    xbar, ybar, zbar = m["xbar"], m["ybar"], m["zbar"]
    xpbar, ypbar, vxbar, vybar, vzbar = m["xpbar"], m["ypbar"], m["vxbar"], m["vybar"], m["vzbar"]
    delxsq = m["xsqbar"] - xbar * xbar
    delxxp = m["xxpbar"] - xbar * xpbar
    delxpsq = m["xpsqbar"] - xpbar * xpbar
    delxvx = m["xvxbar"] - xbar * vxbar
    delvxsq = m["vxsqbar"] - vxbar ** 2
    delysq = m["ysqbar"] - ybar * ybar
    delyyp = m["yypbar"] - ybar * ypbar
    delypsq = m["ypsqbar"] - ypbar * ypbar
    delyvy = m["yvybar"] - ybar * vybar
    delvysq = m["vysqbar"] - vybar ** 2
    delxy = m["xybar"] - xbar * ybar
    delxyp = m["xypbar"] - xbar * ypbar
    delyxp = m["yxpbar"] - ybar * xpbar
    delxpyp = m["xpypbar"] - xpbar * ypbar
    delzsq = m["zsqbar"] - zbar ** 2
    delvzsq = m["vzsqbar"] - vzbar ** 2
    delzvz = m["zvzbar"] - zbar * vzbar
    clighti = 1. / clight
    pos = lambda a: np.maximum(0., a)
    m["xrms"] = np.sqrt(pos(delxsq))
    m["yrms"] = np.sqrt(pos(delysq))
    m["zrms"] = np.sqrt(pos(delzsq))
    m["rrms"] = np.sqrt(m["xrms"] ** 2 + m["yrms"] ** 2)
    m["xprms"] = np.sqrt(pos(delxpsq))
    m["yprms"] = np.sqrt(pos(delypsq))
    m["vxrms"] = np.sqrt(pos(delvxsq))
    m["vyrms"] = np.sqrt(pos(delvysq))
    m["vzrms"] = np.sqrt(pos(delvzsq))
    m["epsx"] = 4. * np.sqrt(pos(delxsq * delxpsq - delxxp ** 2))
    m["epsy"] = 4. * np.sqrt(pos(delysq * delypsq - delyyp ** 2))
    m["epsnx"] = 4. * np.sqrt(pos(delxsq * delvxsq - delxvx ** 2)) * clighti * 1.e6
    m["epsny"] = 4. * np.sqrt(pos(delysq * delvysq - delyvy ** 2)) * clighti * 1.e6
    m["epsnz"] = 4. * np.sqrt(pos(delzsq * delvzsq - delzvz ** 2)) * clighti
    tr = 4. * ((delxsq + delysq) * (delxpsq + delypsq) - (delxxp + delyyp) ** 2 - (delxyp - delyxp) ** 2)
    m["epsr"] = np.sqrt(pos(tr))
    tg = 0.5 * (m["epsx"] ** 2 + m["epsy"] ** 2) + 16 * (delxy * delxpyp - delxyp * delyxp)
    m["epsg"] = np.sqrt(pos(tg))
    return {k + suffix: v for k, v in m.items()}


def zmoment_sums_host(p, po, dt, zmmntmin, zmmntmax, nzmmnt, zbeam=0.0, dtscale=1.0, zmmntdtextmax=1e36):
    """The same sums as wg_zmoments with numpy, for checks on small inputs:
    p holds x, y, z, ux, uy, uz, gaminv; po the velocities dt earlier."""
    live = p["gaminv"] != 0
    x, y, z = (p[k][live] for k in ("x", "y", "z"))
    ux, uy, uz, gi = (p[k][live] for k in ("ux", "uy", "uz", "gaminv"))
    uxo, uyo, uzo = (po[k][live] for k in ("ux", "uy", "uz"))

    def terms(qx, qy, qz, px, py, pz, w, vz):
        v = 1. / (vz + SMALLPOS)
        t = np.zeros((len(qx), 33))
        t[:, 0] = w
        t[:, 1], t[:, 2], t[:, 3] = qx * w, qy * w, qz * w
        t[:, 6], t[:, 7], t[:, 8] = px * w, py * w, pz * w
        t[:, 9] = qx * qy * w
        t[:, 11], t[:, 12], t[:, 13] = qx * qx * w, qy * qy * w, qz * qz * w
        t[:, 16], t[:, 17], t[:, 18] = px * px * w, py * py * w, pz * pz * w
        t[:, 21], t[:, 24], t[:, 25] = qz * pz * w, qx * pz * w, qy * pz * w
        t[:, 26], t[:, 27] = px * pz * w, py * pz * w
        t[:, 4], t[:, 5] = px * v * w, py * v * w
        t[:, 10] = px * py * (v * v) * w
        t[:, 14], t[:, 15] = (px * v) * (px * v) * w, (py * v) * (py * v) * w
        t[:, 19], t[:, 20] = qx * px * v * w, qy * py * v * w
        t[:, 22], t[:, 23] = qx * py * v * w, qy * px * v * w
        t[:, 28], t[:, 29], t[:, 30], t[:, 31] = qx * px * w, qy * py * w, qx * py * w, qy * px * w
        t[:, 32] = px * py * w
        return t

    g = terms(x, y, z, ux, uy, uz, np.ones(len(x)), uz).sum(axis=0)
    zm = np.zeros((nzmmnt + 1, 33))
    dzm = (zmmntmax - zmmntmin) / nzmmnt
    dzmi = 1. / dzm
    zr = z - zbeam
    inr = ~((zr < zmmntmin) | (zr >= zmmntmax))
    iz = ((z - zbeam - zmmntmin) * dzmi).astype(np.int64)
    iz[iz == nzmmnt] = nzmmnt - 1
    vzgi = 1. / (uz * gi + SMALLPOS)
    for side in (0, 1):
        dtx = ((iz + side) * dzm - z + zbeam + zmmntmin) * vzgi
        dtx = np.maximum(-zmmntdtextmax * dt, np.minimum(zmmntdtextmax * dt, dtx))
        px = ux * (1. + dtx / dt) - uxo * dtx / dt
        py = uy * (1. + dtx / dt) - uyo * dtx / dt
        pz = uz * (1. + dtx / dt) - uzo * dtx / dt
        qx, qy, qz = x + ux * dtx * gi, y + uy * dtx * gi, z + uz * dtx * gi
        w = ((1. - (z - zbeam - zmmntmin) * dzmi + iz) if side == 0 else ((z - zbeam - zmmntmin) * dzmi - iz)) * dtscale
        t = terms(qx, qy, qz, px, py, pz, w, pz)
        np.add.at(zm, iz[inr] + side, t[inr])
    return g, zm
