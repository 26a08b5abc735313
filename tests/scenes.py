"""Seeded synthetic dam-break block scenes (test-side description).

A block scene is an nx-by-ny fluid lattice at spacing dx anchored at the
origin, each coordinate jittered uniformly by +/- jitter*dx from
std::mt19937_64{seed}, inside a [0, length]^2 tank whose floor and side walls
are three rows of boundary particles at the same spacing. Kernel support is
``support_ratio * dx`` (the reference's own default scene uses a support
equal to its lattice spacing). The product builds the same scenes in C++
(emerald_b200/csrc/host/scene.cpp); tests compare both.
"""
import numpy as np

F = np.float32
TPS_DEFAULT = 23520000  # 3/90 s in flicks (emerald/sph2d_box/parameters.h:14)


def walls(dx, length=1.0, layers=3):
    dx = F(dx)
    length = F(length)
    n = int(round(float(length) / float(dx)))
    pts = []
    for k in range(layers):
        off = (F(k) + F(0.5)) * dx
        for i in range(-layers, n + layers):
            pts.append(((F(i) + F(0.5)) * dx, -off))
        for j in range(n):
            pts.append((-off, (F(j) + F(0.5)) * dx))
        for j in range(n):
            pts.append((length + off, (F(j) + F(0.5)) * dx))
    return np.array(pts, np.float32)


def lattice_template(kernel_w, kernel_grad_w, length_fn, support, dx, rho0, dt):
    """Mass per particle and PCISPH denominator of an unjittered square lattice
    at spacing dx, in the form of emerald/sph2d_box/config.cpp:16-132."""
    h = F(support)
    dx = F(dx)
    reach = int(np.ceil(2.0 * float(h) / float(dx))) + 1
    muchness = F(0.0)
    gsum = np.zeros(2, np.float32)
    gdot = F(0.0)
    for j in range(-reach, reach + 1):
        for i in range(-reach, reach + 1):
            px = F(i) * dx
            py = F(j) * dx
            ddx = F(0.0) - px
            ddy = F(0.0) - py
            r = F(length_fn(ddx, ddy))
            w = F(kernel_w(r, h))
            if w > F(0.0):
                muchness = F(muchness + w)
            g = kernel_grad_w(ddx, ddy, h)
            gsum[0] = F(gsum[0] + g[0])
            gsum[1] = F(gsum[1] + g[1])
            gdot = F(gdot + F(F(g[0] * g[0]) + F(g[1] * g[1])))
    mass = F(F(rho0) / muchness)
    beta = F(F(2.0) * F(F(F(dt) / muchness) * F(F(dt) / muchness)))
    denom = F(beta * F(F(F(gsum[0] * gsum[0]) + F(gsum[1] * gsum[1])) + gdot))
    return mass, denom
