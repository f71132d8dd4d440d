"""An independent float32 numpy restatement of the reference's stencil passes.

Written from the WGSL again (src/engine/simulation/shaders/passes/*.wgsl.ts),
separately from the C++ oracle, to cross-check it bit for bit on the passes that
use only +, -, *, / and sqrt. Arrays are indexed [z, y, x]. numpy evaluates each
float32 operation with IEEE round-to-nearest and never fuses a multiply-add, so
the same operation order gives the same bits.
"""
from __future__ import annotations

import numpy as np

F = np.float32


def mix(a, b, t):
    return a * (F(1) - t) + b * t


def clampv(x, lo, hi):
    # min(max(x, lo), hi) with the comparison order of the oracle and the kernels
    x = np.where(x < lo, lo, x)
    return np.where(hi < x, hi, x)


def smoothstep(e0, e1, x):
    t = clampv((x - F(e0)) / (F(e1) - F(e0)), F(0), F(1))
    return t * t * (F(3) - F(2) * t)


def length3(x, y, z):
    return np.sqrt(x * x + y * y + z * z)


def boundary_mask(shape):
    d, h, w = shape
    m = np.zeros(shape, bool)
    m[0, :, :] = m[-1, :, :] = True
    m[:, 0, :] = m[:, -1, :] = True
    m[:, :, 0] = m[:, :, -1] = True
    return m


def jacobi(div, p):
    """pressure-jacobi.wgsl.ts:15-36."""
    out = np.zeros_like(p)
    s = p[1:-1, 1:-1, 2:] + p[1:-1, 1:-1, :-2]
    s = s + p[1:-1, 2:, 1:-1]
    s = s + p[1:-1, :-2, 1:-1]
    s = s + p[2:, 1:-1, 1:-1]
    s = s + p[:-2, 1:-1, 1:-1]
    out[1:-1, 1:-1, 1:-1] = (s - div[1:-1, 1:-1, 1:-1]) / F(6)
    return out


def divergence(vx, vy, vz):
    """compute-divergence.wgsl.ts:22-42."""
    out = np.zeros_like(vx)
    dx = vx[1:-1, 1:-1, 2:] - vx[1:-1, 1:-1, :-2]
    dy = vy[1:-1, 2:, 1:-1] - vy[1:-1, :-2, 1:-1]
    dz = vz[2:, 1:-1, 1:-1] - vz[:-2, 1:-1, 1:-1]
    out[1:-1, 1:-1, 1:-1] = (dx + dy + dz) * F(0.5)
    return out


def project(vx, vy, vz, p):
    """project-velocity.wgsl.ts:21-43."""
    ox, oy, oz = np.zeros_like(vx), np.zeros_like(vy), np.zeros_like(vz)
    gx = (p[1:-1, 1:-1, 2:] - p[1:-1, 1:-1, :-2]) * F(0.5)
    gy = (p[1:-1, 2:, 1:-1] - p[1:-1, :-2, 1:-1]) * F(0.5)
    gz = (p[2:, 1:-1, 1:-1] - p[:-2, 1:-1, 1:-1]) * F(0.5)
    i = (slice(1, -1),) * 3
    ox[i] = vx[i] - gx
    oy[i] = vy[i] - gy
    oz[i] = vz[i] - gz
    return ox, oy, oz


def curl(vx, vy, vz):
    """compute-vorticity.wgsl.ts:23-50 -> (wx, wy, wz, |w|)."""
    shp = vx.shape
    wx, wy, wz, wm = (np.zeros(shp, F) for _ in range(4))
    i = (slice(1, -1),) * 3

    def dxp(a):
        return a[1:-1, 1:-1, 2:], a[1:-1, 1:-1, :-2]

    def dyp(a):
        return a[1:-1, 2:, 1:-1], a[1:-1, :-2, 1:-1]

    def dzp(a):
        return a[2:, 1:-1, 1:-1], a[:-2, 1:-1, 1:-1]

    y1, y0 = dyp(vz)
    z1, z0 = dzp(vy)
    cx = ((y1 - y0) - (z1 - z0)) * F(0.5)
    z1, z0 = dzp(vx)
    x1, x0 = dxp(vz)
    cy = ((z1 - z0) - (x1 - x0)) * F(0.5)
    x1, x0 = dxp(vy)
    y1, y0 = dyp(vx)
    cz = ((x1 - x0) - (y1 - y0)) * F(0.5)
    wx[i], wy[i], wz[i] = cx, cy, cz
    wm[i] = length3(cx, cy, cz)
    return wx, wy, wz, wm


def confinement(wx, wy, wz, wm, d, t, r, vx, vy, vz, params):
    """apply-vorticity-confinement.wgsl.ts:30-66 -> (vx, vy, vz, |F|)."""
    i = (slice(1, -1),) * 3
    gx = (wm[1:-1, 1:-1, 2:] - wm[1:-1, 1:-1, :-2]) * F(0.5)
    gy = (wm[1:-1, 2:, 1:-1] - wm[1:-1, :-2, 1:-1]) * F(0.5)
    gz = (wm[2:, 1:-1, 1:-1] - wm[:-2, 1:-1, 1:-1]) * F(0.5)
    gl = length3(gx, gy, gz)
    gl = np.where(gl < F(0.0001), F(0.0001), gl)
    nx, ny, nz = gx / gl, gy / gl, gz / gl
    hot = clampv(t[i] + r[i] * F(0.85), F(0), F(1))
    vm = params["vmask"]
    mask = clampv(F(vm[0]) + smoothstep(0.02, 0.38, wm[i]) * F(vm[1]) + smoothstep(0.04, 0.7, hot) * F(vm[2])
                  + smoothstep(0.04, 0.65, d[i]) * F(vm[3]), F(0), F(4))
    k = F(params["vorticity_strength"])
    fx = (ny * wz[i] - nz * wy[i]) * k * mask * F(1.45)
    fy = (nz * wx[i] - nx * wz[i]) * k * mask * F(1.45)
    fz = (nx * wy[i] - ny * wx[i]) * k * mask * F(1.45)
    dxv = F(params["dx"])
    lim = F(80.0) / (dxv if dxv >= F(0.001) else F(0.001))
    dt = F(params["dt"])
    ox, oy, oz = vx.copy(), vy.copy(), vz.copy()
    ox[i] = clampv(vx[i] + fx * dt, -lim, lim)
    oy[i] = clampv(vy[i] + fy * dt, -lim, lim)
    oz[i] = clampv(vz[i] + fz * dt, -lim, lim)
    fm = np.zeros_like(vx)
    fm[i] = length3(fx, fy, fz)
    return ox, oy, oz, fm


def restrict(div_f, coarse_shape):
    """pressure-restriction.wgsl.ts:27-50."""
    cd, ch, cw = coarse_shape
    fd, fh, fw = div_f.shape
    out = np.zeros(coarse_shape, F)
    z, y, x = np.meshgrid(np.arange(1, cd - 1), np.arange(1, ch - 1), np.arange(1, cw - 1), indexing="ij")
    s = np.zeros(z.shape, F)
    for dz in range(2):
        for dy in range(2):
            for dx in range(2):
                sz = np.minimum(2 * z + dz, fd - 1)
                sy = np.minimum(2 * y + dy, fh - 1)
                sx = np.minimum(2 * x + dx, fw - 1)
                s = s + div_f[sz, sy, sx]
    out[1:-1, 1:-1, 1:-1] = s * F(0.125)
    return out


def trilinear(field, pz, py, px):
    """sampling-scalar.wgsl.ts:11-34 at float32 positions (arrays)."""
    d, h, w = field.shape
    mxp, myp, mzp = F(w - 1), F(h - 1), F(d - 1)

    def cl(p, hi):
        p = np.where(~(p > F(0)), F(0), p)
        return np.where(p < hi, p, hi)

    cx, cy, cz = cl(px, mxp), cl(py, myp), cl(pz, mzp)
    fx, fy, fz = np.floor(cx), np.floor(cy), np.floor(cz)
    bx, by, bz = fx.astype(np.int64), fy.astype(np.int64), fz.astype(np.int64)
    ux, uy, uz = np.minimum(bx + 1, w - 1), np.minimum(by + 1, h - 1), np.minimum(bz + 1, d - 1)
    tx, ty, tz = cx - fx, cy - fy, cz - fz
    x00 = mix(field[bz, by, bx], field[bz, by, ux], tx)
    x10 = mix(field[bz, uy, bx], field[bz, uy, ux], tx)
    x01 = mix(field[uz, by, bx], field[uz, by, ux], tx)
    x11 = mix(field[uz, uy, bx], field[uz, uy, ux], tx)
    return mix(mix(x00, x10, ty), mix(x01, x11, ty), tz)


def prolong(coarse_p, fine_pa):
    """pressure-prolongation.wgsl.ts:29-44."""
    out = fine_pa.copy()
    fd, fh, fw = fine_pa.shape
    z, y, x = np.meshgrid(np.arange(fd, dtype=F), np.arange(fh, dtype=F), np.arange(fw, dtype=F), indexing="ij")
    pz = (z + F(0.5)) * F(0.5) - F(0.5)
    py = (y + F(0.5)) * F(0.5) - F(0.5)
    px = (x + F(0.5)) * F(0.5) - F(0.5)
    s = trilinear(coarse_p, pz, py, px)
    out = out + s
    out[boundary_mask(out.shape)] = F(0)
    return out


def advect_velocity(vx, vy, vz, dt):
    """advect-velocity-semilagrangian.wgsl.ts:23-41 (no clamp: fields within the limit)."""
    d, h, w = vx.shape
    z, y, x = np.meshgrid(np.arange(d, dtype=F), np.arange(h, dtype=F), np.arange(w, dtype=F), indexing="ij")
    cx, cy, cz = x + F(0.5), y + F(0.5), z + F(0.5)
    dt = F(dt)
    s = [trilinear(c, cz - F(0.5), cy - F(0.5), cx - F(0.5)) for c in (vx, vy, vz)]
    bx, by, bz = cx - s[0] * dt, cy - s[1] * dt, cz - s[2] * dt
    damp = F(1) - dt * F(0.025)
    out = [trilinear(c, bz - F(0.5), by - F(0.5), bx - F(0.5)) * damp for c in (vx, vy, vz)]
    m = boundary_mask(vx.shape)
    for o in out:
        o[m] = F(0)
    return out


def brick_flags(d, t, r):
    """compute-active-bricks.wgsl.ts:24-79 (flags cleared first)."""
    D, H, W = d.shape
    bx, by, bz = -(-W // 8), -(-H // 8), -(-D // 8)
    e = d + t * F(0.7) + r * F(0.9)
    flags = np.zeros((bz, by, bx), np.uint32)
    for k in range(bz):
        for j in range(by):
            for i in range(bx):
                z0, y0, x0 = 8 * k, 8 * j, 8 * i
                samp = e[z0:z0 + 8:2, y0:y0 + 8:2, x0:x0 + 8:2]
                ce = e[min(z0 + 4, D - 1), min(y0 + 4, H - 1), min(x0 + 4, W - 1)]
                peak = max(F(0), samp.max() if samp.size else F(0), ce)
                active = bool((samp > F(0.012)).any()) or ce > F(0.012)
                if not active:
                    continue
                rad = 1 if (peak > F(0.05) or ce > F(0.035)) else 0
                flags[max(k - rad, 0):min(k + rad, bz - 1) + 1, max(j - rad, 0):min(j + rad, by - 1) + 1,
                      max(i - rad, 0):min(i + rad, bx - 1) + 1] = 1
    return flags.ravel()
