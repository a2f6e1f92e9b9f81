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
- ``LayeredPlaneWave``: the same for a stack of layers over the
  half-space (frequency-domain layer matrices; FK3D's job);
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


def injection_arrays(db, wave, nt, dt, np_resamp=1, k0=0):
    """Velocity and traction samples ``[nt, nf*25, 3]`` at the absorbing face
    points, sample ``k`` at time ``(k + k0) * np_resamp * dt``."""
    xyz, nrm = face_points(db)
    t = (np.arange(nt) + k0) * np_resamp * dt
    return wave.velocity(xyz, t), wave.traction(xyz, nrm, t)


class LayeredPlaneWave:
    """P or SV plane wave incident from the half-space below a stack of
    homogeneous layers with a free surface on top: the incident field of
    FK injection (what SPECFEM's FK3D computes for
    couple_with_injection_prepare_boundary_fwat, fk_coupling.f90:71-297).

    ``vp, vs, rho``: per layer from the top, the last entry the half-space;
    ``h``: thicknesses of the finite layers (``len(vp) - 1`` of them).  The
    ray parameter is ``sin(theta) / v`` of the half-space (fk_coupling.f90:
    150-156).  The incident wave's displacement time function is the
    Gaussian ``exp(-(pi f0 tau)^2)``, ``tau = 0`` passing ``x0`` (in the
    half-space) at ``t0``.

    Per frequency the up- and down-going P and SV amplitudes of every layer
    solve the free-surface and interface continuity conditions of
    displacement and traction (a (4N-2)-square system for N layers, each
    wave's phase referred to the layer edge it travels away from, so that
    evanescent waves stay bounded).  Fields at a point are the sums over
    its layer's waves, back in time by an inverse real FFT over the band
    where the Gaussian's spectrum exceeds 1e-14 of its peak.
    """

    def __init__(self, vp, vs, rho, h, theta_deg, phi_deg, wave="P", f0=0.2, t0=5.0,
                 x0=(0.0, 0.0, -1.0e4), z_top=0.0, amplitude=1.0):
        self.vp = np.asarray(vp, np.float64)
        self.vs = np.asarray(vs, np.float64)
        self.rho = np.asarray(rho, np.float64)
        self.h = np.asarray(h, np.float64).reshape(-1)
        n = self.vp.size
        if not (self.vs.size == self.rho.size == n and self.h.size == n - 1):
            raise ValueError("vp, vs, rho need one entry per layer and h one per finite layer")
        if wave not in ("P", "SV"):
            raise ValueError("wave must be 'P' or 'SV'")
        self.n = n
        self.mu = self.rho * self.vs ** 2
        self.lam = self.rho * self.vp ** 2 - 2.0 * self.mu
        self.wave = wave
        v_in = self.vp[-1] if wave == "P" else self.vs[-1]
        self.p = np.sin(np.deg2rad(theta_deg)) / v_in
        if self.p * self.vp[-1] >= 1.0:
            raise ValueError("the half-space's reflected P wave would be evanescent")
        ph = np.deg2rad(phi_deg)
        self.eh = np.array([np.cos(ph), np.sin(ph), 0.0])
        self.f0, self.t0, self.z_top = float(f0), float(t0), float(z_top)
        self.x0 = np.asarray(x0, np.float64)
        self.amp = float(amplitude)
        # layer edges from the top: z_edge[j] top of layer j, z_edge[j+1] its bottom
        self.z_edge = self.z_top - np.concatenate([[0.0], np.cumsum(self.h)])
        if self.x0[2] > self.z_edge[-1]:
            raise ValueError("x0 must lie in the half-space")

    # vertical slowness; an evanescent wave takes eta = -i kappa, so that
    # with omega > 0 it decays away from its reference edge
    def _eta(self, v):
        x = 1.0 / v ** 2 - self.p ** 2
        return np.sqrt(x) + 0j if x >= 0 else -1j * np.sqrt(-x)

    def _waves(self, j):
        """(q, d_h, d_z) of the 4 waves of layer j: up P, down P, up S, down S."""
        p = self.p
        ea, eb = self._eta(self.vp[j]), self._eta(self.vs[j])
        a, b = self.vp[j], self.vs[j]
        return [(ea, a * p, a * ea), (-ea, a * p, -a * ea),
                (eb, b * eb, -b * p), (-eb, -b * eb, -b * p)]

    def _ref(self, j, k):
        """Reference depth of wave k of layer j: up waves the layer bottom,
        down waves the layer top; the incident wave x0's depth."""
        if j == self.n - 1:
            return self.x0[2] if k in (0, 2) else self.z_edge[-1]
        return self.z_edge[j + 1] if k in (0, 2) else self.z_edge[j]

    def _bvec(self, j, k, w, z):
        """(u_h, u_z, s_hz, s_zz) of unit amplitude wave k of layer j at z."""
        q, dh, dz = self._waves(j)[k]
        e = np.exp(-1j * w * q * (z - self._ref(j, k)))
        lam, mu, p = self.lam[j], self.mu[j], self.p
        shz = -1j * w * mu * (p * dz + q * dh)
        szz = -1j * w * (lam * (p * dh + q * dz) + 2.0 * mu * q * dz)
        return e * np.array([dh, dz, shz, szz])

    def _solve(self, w):
        """Amplitudes [n, 4] (half-space: incident up wave 1, its other up
        wave 0) at angular frequency w > 0."""
        n = self.n
        inc = 0 if self.wave == "P" else 2
        nu = 4 * (n - 1) + 2
        idx = {}
        c = 0
        for j in range(n - 1):
            for k in range(4):
                idx[(j, k)] = c
                c += 1
        idx[(n - 1, 1)] = c
        idx[(n - 1, 3)] = c + 1
        M = np.zeros((nu, nu), np.complex128)
        rhs = np.zeros(nu, np.complex128)
        row = 0

        def add(j, z, sign, rows):
            for k in range(4):
                b = sign * self._bvec(j, k, w, z)[rows]
                if (j, k) in idx:
                    M[row:row + len(rows), idx[(j, k)]] += b
                elif j == n - 1 and k == inc:
                    rhs[row:row + len(rows)] -= b
        add(0, self.z_top, 1.0, [2, 3])
        row += 2
        for j in range(n - 1):
            z = self.z_edge[j + 1]
            add(j, z, 1.0, [0, 1, 2, 3])
            add(j + 1, z, -1.0, [0, 1, 2, 3])
            row += 4
        scale = np.abs(M).max(axis=1)
        scale[scale == 0] = 1.0
        x = np.linalg.solve(M / scale[:, None], rhs / scale)
        A = np.zeros((n, 4), np.complex128)
        for (j, k), i in idx.items():
            A[j, k] = x[i]
        A[n - 1, inc] = 1.0
        return A

    def _layer(self, z):
        j = np.searchsorted(-self.z_edge[1:], -np.asarray(z), side="left")
        return np.minimum(j, self.n - 1)

    def _fields(self, xyz, t, normals=None, what="u"):
        xyz = np.asarray(xyz, np.float64).reshape(-1, 3)
        t = np.asarray(t, np.float64)
        dt = t[1] - t[0] if t.size > 1 else 1.0
        if t.size > 1 and not np.allclose(np.diff(t), dt, rtol=1e-9, atol=1e-12):
            raise ValueError("t must be uniformly sampled")
        # FFT period long enough that nothing wraps into the window
        span = t[-1] - t[0]
        reach = abs(self.t0) + 3.0 / self.f0 + np.ptp(xyz, axis=0).sum() / self.vs.min() \
            + (self.z_top - self.x0[2]) / self.vs.min() + abs(t[0])
        nfft = 1 << int(np.ceil(np.log2((2.0 * (span + reach)) / dt + 2)))
        w = 2.0 * np.pi * np.fft.rfftfreq(nfft, dt)
        a = np.pi * self.f0
        G = (np.sqrt(np.pi) / a) * np.exp(-(w / (2.0 * a)) ** 2) * self.amp
        keep = np.nonzero(G > 1e-14 * G[0])[0]
        out = np.zeros((t.size, xyz.shape[0], 3))
        lay = self._layer(xyz[:, 2])
        dxh = (xyz - self.x0) @ self.eh
        nrm = None if normals is None else np.asarray(normals, np.float64).reshape(-1, 3)
        spec = np.zeros((w.size, xyz.shape[0], 3), np.complex128)
        for i in keep:
            wi = w[i] if w[i] > 0 else 1e-6 * w[1]
            A = self._solve(wi)
            base = G[i] * np.exp(-1j * wi * (self.p * dxh + self.t0 - t[0]))
            for j in np.unique(lay):
                sel = lay == j
                z = xyz[sel, 2]
                acc = np.zeros((sel.sum(), 3), np.complex128)
                for k, (q, dh, dz) in enumerate(self._waves(j)):
                    if A[j, k] == 0:
                        continue
                    e = A[j, k] * np.exp(-1j * wi * q * (z - self._ref(j, k)))
                    d = dh * self.eh + dz * np.array([0.0, 0.0, 1.0])
                    if what == "u":
                        acc += e[:, None] * d[None, :]
                    elif what == "v":
                        acc += (1j * wi * e)[:, None] * d[None, :]
                    else:
                        s = self.p * self.eh + q * np.array([0.0, 0.0, 1.0])
                        nn = nrm[sel]
                        vec = (self.lam[j] * (d @ s)) * nn + self.mu[j] * (
                            np.outer(nn @ s, d) + np.outer(nn @ d, s))
                        acc += (-1j * wi * e)[:, None] * vec
                spec[i, sel] = base[sel, None] * acc
        return np.fft.irfft(spec, n=nfft, axis=0)[: t.size] / dt

    def displacement(self, xyz, t):
        return self._fields(xyz, t, what="u")

    def velocity(self, xyz, t):
        return self._fields(xyz, t, what="v")

    def traction(self, xyz, normals, t):
        return self._fields(xyz, t, normals, what="t")


def read_fkmodel(path):
    """The keyword file the reference names ``src_rec/FKmodel_<event>``
    (``read_fk_model``, src/shared/fk_coupling.f90:12-59): ``NLAYER n``,
    ``LAYER i rho vp vs ztop`` per layer from the top (the last one the
    half-space, its ``ztop`` the half-space's top), ``INCIDENT_WAVE p|sv``,
    ``BACK_AZIMUTH`` and ``TAKE_OFF`` in degrees, ``FREQUENCY_MAX``,
    ``TIME_WINDOW``, and optionally ``FREQUENCY_SAMPLING``, ``AMPLITUDE``,
    ``ORIGIN_WAVEFRONT x y z`` and ``ORIGIN_TIME``.  ``#`` starts a
    comment.  Returns a dict with those values (layers as arrays)."""
    d = {"layers": {}}
    with open(path) as f:
        for raw in f:
            line = raw.split("#", 1)[0].strip()
            if not line:
                continue
            key, *vals = line.split()
            key = key.upper()
            if key == "LAYER":
                i, rho, vp, vs, ztop = vals[:5]
                d["layers"][int(i)] = (float(rho), float(vp), float(vs), float(ztop))
            elif key == "NLAYER":
                d["nlayer"] = int(vals[0])
            elif key == "INCIDENT_WAVE":
                d["wave"] = vals[0].upper()
            elif key == "ORIGIN_WAVEFRONT":
                d["origin_wavefront"] = tuple(float(v) for v in vals[:3])
            elif key in ("BACK_AZIMUTH", "TAKE_OFF", "FREQUENCY_MAX", "FREQUENCY_SAMPLING",
                         "TIME_WINDOW", "AMPLITUDE", "ORIGIN_TIME"):
                d[key.lower()] = float(vals[0])
    n = d.get("nlayer", len(d["layers"]))
    if sorted(d["layers"]) != list(range(1, n + 1)):
        raise ValueError(f"{path}: LAYER lines 1..{n} expected, got {sorted(d['layers'])}")
    lay = np.array([d["layers"][i] for i in range(1, n + 1)], np.float64)
    if np.any(np.diff(lay[:, 3]) >= 0):
        raise ValueError(f"{path}: layer tops must decrease downward")
    d["rho"], d["vp"], d["vs"], d["ztop"] = lay[:, 0], lay[:, 1], lay[:, 2], lay[:, 3]
    for k in ("wave", "back_azimuth", "take_off"):
        if k not in d:
            raise ValueError(f"{path}: {k.upper()} missing")
    if d["wave"] not in ("P", "SV"):
        raise ValueError(f"{path}: INCIDENT_WAVE must be p or sv")
    return d


def plane_wave_from_fkmodel(fk, x0=None, t0=None):
    """``LayeredPlaneWave`` of an ``read_fkmodel`` dict.

    - The propagation azimuth measured from +x (east) counter-clockwise is
      ``-90 - BACK_AZIMUTH`` degrees (a wave from the back azimuth travels
      the opposite way).
    - The layer thicknesses are the differences of the layer tops; the free
      surface is the first layer's top.
    - ``FREQUENCY_MAX`` sets the Gaussian time function's ``f0``.  The
      reference's FK code (absent here) defines its own wavelet.
    - ``ORIGIN_WAVEFRONT`` and ``ORIGIN_TIME`` give ``x0`` and ``t0`` unless
      passed here; without either the call fails.
    """
    if x0 is None:
        if "origin_wavefront" not in fk:
            raise ValueError("no ORIGIN_WAVEFRONT in the file: pass x0")
        x0 = fk["origin_wavefront"]
    if t0 is None:
        t0 = fk.get("origin_time", 0.0)
    h = -np.diff(fk["ztop"])
    return LayeredPlaneWave(fk["vp"], fk["vs"], fk["rho"], h, fk["take_off"],
                            -90.0 - fk["back_azimuth"], fk["wave"],
                            f0=fk.get("frequency_max", 0.2), t0=t0, x0=x0,
                            z_top=float(fk["ztop"][0]), amplitude=fk.get("amplitude", 1.0))
