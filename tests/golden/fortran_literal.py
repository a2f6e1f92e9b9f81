"""Line-by-line transcriptions of the reference's measurement loops.

Pure-Python, 1-based index arithmetic kept as written in the Fortran, used
only to pin the vectorised restatements in ``oracle/oracle.py`` and to make
the golden vectors in this directory:

* ``simpson``      src/shared/utils.f90:1635-1663
* ``window_taper`` src/shared/signal.f90:419-491
* ``calc_adjoint_source`` (L2, one window)
                   src/preproc/adjoint_sources/waveform_misfit.f90:15-64
"""
import math


def simpson(y, dx):
    n = len(y)
    m = n
    if m < 2:
        return 0.0
    if m % 2 == 0:
        s = y[1 - 1] + y[n - 1 - 1]
        for i in range(2, n - 2 + 1, 2):
            s = s + 4.0 * y[i - 1] + 2.0 * y[i + 1 - 1]
        return (dx / 3.0) * s + 0.5 * dx * (y[n - 1 - 1] + y[n - 1])
    s = y[1 - 1] + y[n - 1]
    for i in range(2, n - 1 + 1, 2):
        s = s + 4.0 * y[i - 1]
    for i in range(3, n - 2 + 1, 2):
        s = s + 2.0 * y[i - 1]
    return (dx / 3.0) * s


def window_taper(signal, taper_percentage, itaper_type):
    sig = list(signal)
    npts = len(sig)
    if taper_percentage in (0.0, 1.0):
        frac = int(npts * taper_percentage / 2.0)
    else:
        frac = int(npts * taper_percentage / 2.0 + 0.5)
    idx1 = frac
    idx2 = npts - frac
    if frac > 0:
        def first(i):
            x = float(i - 1)
            den = 2 * frac - 1
            if itaper_type == 1:
                return 0.5 - 0.5 * math.cos(2.0 * math.pi * x / den)
            if itaper_type == 2:
                return 0.54 - 0.46 * math.cos(2.0 * math.pi * x / den)
            if itaper_type == 3:
                return math.cos(math.pi * x / den - math.pi / 2.0) ** 1.0
            return 1.0 - math.cos(math.pi * x / den) ** 10.0

        def last(i):
            x = float(frac + i - 1)
            den = 2 * frac - 1
            if itaper_type == 1:
                return 0.5 - 0.5 * math.cos(2.0 * math.pi * x / den)
            if itaper_type == 2:
                return 0.54 - 0.46 * math.cos(2.0 * math.pi * x / den)
            if itaper_type == 3:
                return math.cos(math.pi * x / den - math.pi / 2.0) ** 1.0
            return 1.0 - math.cos(math.pi * x / den) ** 10.0

        for i in range(1, frac + 1):
            sig[i - 1] = sig[i - 1] * first(i)
        for i in range(1, frac + 1):
            sig[idx2 + i - 1] = sig[idx2 + i - 1] * last(i)
    _ = idx1
    return sig


def l2_adjoint_source(syn, dat, dt, taper_percentage, itaper_type):
    """One full-record window: returns (misfit, adjoint source)."""
    s = window_taper(syn, taper_percentage, itaper_type)
    d = window_taper(dat, taper_percentage, itaper_type)
    adj_tw = [a - b for a, b in zip(s, d)]
    adj_tw = window_taper(adj_tw, taper_percentage, itaper_type)
    misfit = 0.5 * simpson([(a - b) ** 2 for a, b in zip(s, d)], dt)
    return misfit, adj_tw
