"""Incident wavefields for FK injection on the absorbing faces.

The reference injects a teleseismic plane wave through the absorbing
boundary: ``couple_with_injection_prepare_boundary_fwat``
(src/shared/fk_coupling.f90:71-297) has SPECFEM's FK3D compute the velocity
and traction of the layered model's plane-wave response at every absorbing
face point (``Veloc_FK``, ``Tract_FK``), and the solver's Stacey routine
absorbs the velocity relative to that field and adds its traction
(``sem_set_injection``).

This module gives the one-layer case in closed form: a P or SV plane wave
of horizontal slowness ``p = sin(theta) / v`` and azimuth ``phi`` incident
from below on a homogeneous half-space with a free surface at ``z_top``,
plus the reflected P and SV waves.  Their amplitudes follow from zero
traction at the surface, solved as a 2x2 system (no polarity convention to
carry).  The displacement time function is a Gaussian of characteristic
frequency ``f0``, ``g(tau) = exp(-(pi f0 tau)^2)``; the incident wave's
``tau = 0`` passes the point ``x0`` at time ``t0`` (the reference's
``xx0, yy0, zz0`` and ``tt0``, fk_coupling.f90:441-484).

Functions:
- ``face_points(db)``: absorbing face points and outward normals, in the
  ``ipt_table`` order of fk_coupling.f90:299-327 (face by face);
- ``HalfspacePlaneWave``: displacement, velocity and traction anywhere;
- ``injection_arrays(db, wave, nt, dt, np_resamp, k0)``: the
  ``[nt, nf*25, 3]`` velocity and traction arrays ``sem_set_injection``
  takes.
"""
from __future__ import annotations

import numpy as np


def face_points(db):
    """xyz and outward normals of the absorbing face points, [nf*25, 3]."""
    ib = np.asarray(db.ibool).reshape(db.nspec, 5, 5, 5)
    ijk = np.asarray(db.abs_ijk)
    e = np.repeat(np.asarray(db.abs_ispec), 25)
    i, j, k = ijk[..., 0].reshape(-1), ijk[..., 1].reshape(-1), ijk[..., 2].reshape(-1)
    ig = ib[e, k, j, i]
    xyz = np.stack([db.xstore[ig], db.ystore[ig], db.zstore[ig]], axis=1).astype(np.float64)
    return xyz, np.asarray(db.abs_normal, np.float64).reshape(-1, 3)


class HalfspacePlaneWave:
    """Incident plus reflected plane waves in a homogeneous half-space."""

    def __init__(self, vp, vs, rho, theta_deg, phi_deg, wave="P", f0=0.2, t0=5.0,
                 x0=(0.0, 0.0, 0.0), z_top=0.0, amplitude=1.0):
        if wave not in ("P", "SV"):
            raise ValueError("wave must be 'P' or 'SV'")
        self.vp, self.vs, self.rho = float(vp), float(vs), float(rho)
        self.mu = rho * vs * vs
        self.lam = rho * vp * vp - 2.0 * self.mu
        th, ph = np.deg2rad(theta_deg), np.deg2rad(phi_deg)
        v_in = vp if wave == "P" else vs
        p = np.sin(th) / v_in
        if p * vp >= 1.0:
            raise ValueError("post-critical incidence: the reflected P wave is evanescent")
        self.f0, self.t0, self.z_top = float(f0), float(t0), float(z_top)
        self.x0 = np.asarray(x0, np.float64)
        eh = np.array([np.cos(ph), np.sin(ph), 0.0])
        ez = np.array([0.0, 0.0, 1.0])
        ea, eb = np.sqrt(1.0 / vp**2 - p * p), np.sqrt(1.0 / vs**2 - p * p)
        cj, sj = eb * vs, p * vs            # cos and sin of the S angle
        ci, si = ea * vp, p * vp            # cos and sin of the P angle
        # (slowness, polarisation) of incident, reflected P, reflected SV
        if wave == "P":
            inc = (p * eh + ea * ez, si * eh + ci * ez)
        else:
            inc = (p * eh + eb * ez, cj * eh - sj * ez)
        rp = (p * eh - ea * ez, si * eh - ci * ez)
        rs = (p * eh - eb * ez, cj * eh + sj * ez)

        def trac_z(w):
            s, d = w
            t = self.mu * (d * s[2] + d[2] * s)
            t[2] += self.lam * (d @ s)
            return np.array([t @ eh, t[2]])

        A = np.stack([trac_z(rp), trac_z(rs)], axis=1)
        r = np.linalg.solve(A, -trac_z(inc))
        self.waves = [(inc[0], inc[1], amplitude), (rp[0], rp[1], amplitude * r[0]),
                      (rs[0], rs[1], amplitude * r[1])]
        # delay of each wave at x: tau = t - t0 - s_inc.(x_s - x0) - s.(x - x_s)
        # with x_s the point of the surface above x, so that all three share
        # the incident phase on the surface
        self.inc_slow = inc[0]

    def _tau(self, xyz, t):
        xyz = np.asarray(xyz, np.float64).reshape(-1, 3)
        xs = xyz.copy()
        xs[:, 2] = self.z_top
        base = (xs - self.x0) @ self.inc_slow                     # [n]
        out = []
        for s, _, _ in self.waves:
            delay = base + (xyz - xs) @ s
            out.append(np.asarray(t, np.float64)[:, None] - self.t0 - delay[None, :])
        return out                                                 # [nt, n] each

    def _g(self, tau, order):
        a = (np.pi * self.f0) ** 2
        e = np.exp(-a * tau * tau)
        if order == 0:
            return e
        return -2.0 * a * tau * e

    def displacement(self, xyz, t):
        """[nt, n, 3]."""
        return sum(amp * self._g(tau, 0)[..., None] * d
                   for (s, d, amp), tau in zip(self.waves, self._tau(xyz, t)))

    def velocity(self, xyz, t):
        return sum(amp * self._g(tau, 1)[..., None] * d
                   for (s, d, amp), tau in zip(self.waves, self._tau(xyz, t)))

    def traction(self, xyz, normals, t):
        """sigma . n, [nt, n, 3]: for u = A d g(t - s.x),
        sigma_ij = -A g' (lambda delta_ij d.s + mu (d_i s_j + d_j s_i))."""
        n = np.asarray(normals, np.float64).reshape(-1, 3)
        out = 0.0
        for (s, d, amp), tau in zip(self.waves, self._tau(xyz, t)):
            sn = n @ s                                             # [n]
            dn = n @ d
            vec = self.lam * (d @ s) * n + self.mu * (np.outer(sn, d) + np.outer(dn, s))
            out = out - amp * self._g(tau, 1)[..., None] * vec[None, :, :]
        return out


def injection_arrays(db, wave: HalfspacePlaneWave, nt, dt, np_resamp=1, k0=0):
    """Velocity and traction samples ``[nt, nf*25, 3]`` at the absorbing face
    points, sample ``k`` at time ``(k + k0) * np_resamp * dt``."""
    xyz, nrm = face_points(db)
    t = (np.arange(nt) + k0) * np_resamp * dt
    return wave.velocity(xyz, t), wave.traction(xyz, nrm, t)
