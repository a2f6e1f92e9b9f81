"""Line-by-line transcriptions of the reference's measurement loops.

Pure-Python, 1-based index arithmetic kept as written in the Fortran, used
only to pin the vectorised restatements in ``oracle/oracle.py`` and to make
the golden vectors in this directory:

* ``simpson``      src/shared/utils.f90:1635-1663
* ``window_taper`` src/shared/signal.f90:419-491
* ``calc_adjoint_source`` (L2, one window)
                   src/preproc/adjoint_sources/waveform_misfit.f90:15-64
* ``invert_hess``  src/postproc/post_processing.f90:333-372 (FP32)
* ``interp1_0``    src/shared/utils.f90:889-910
* ``get_1d_precond``, ``zprecond_gll`` src/postproc/zprecond.f90:11-71 (FP32)
* ``coswin``, ``create_taper``  src/postproc/taper_3D_mod.f90 (FP32)
* ``locate_bissection``, ``interp3``  src/shared/utils.f90:1089-1159,1490-1525
* ``get_nearest_bound_idx``, ``interp3_nearest_simple``  src/shared/utils.f90:
  1262-1325, and ``model_external_values`` (one GLL point)
  src/patch/model_external_values.f90:206-273
* ``project_sem2fd``: compute_interpolation_coeff_FD_SEM + Project_model_
  SEM2FD_grid (src/shared/projection_on_FD_grid_mod_fwat.f90:186-596), one
  slice, regular elements (reference coordinates linear in x, y, z, clamped
  to [-1, 1] as locate_point_in_element's iterations do, :935-1125)
* ``locate_point_in_element`` (:935-1125) with NGNOD = 8 and NUM_ITER = 4,
  and ``project_sem2fd_located`` using it for every element
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


def smooth_sem_pde_cpu(dat_in, ibool, xstore, ystore, zstore, xix_regular,
                       jacobian_regular, sigma_h, sigma_v, distance_min_glob,
                       is_sph, is_cpml=None, nstep=None, irregular_element_number=None,
                       stores=None):
    """CPU branch of ``smooth_sem_pde`` (src/postproc/smooth.f90:7-437), one
    field, CUSTOM_REAL = float32.

    ``dat_in`` is dat(NGLLX,NGLLY,NGLLZ,NSPEC) flattened in Fortran order,
    ``ibool`` the same shape with 1-based global numbers, the stores 1-D.
    Returns the smoothed dat in the same layout and ntstep.  ``nstep``
    replaces ntstep (the regular branch diverges within a few tens of
    steps, so comparisons use a few).  ``irregular_element_number`` [nspec]
    (0 regular, k >= 1 irregular) and ``stores`` = (xixstore, xiystore,
    xizstore, etaxstore, etaystore, etazstore, gammaxstore, gammaystore,
    gammazstore, jacobianstore), each (NGLLX,NGLLY,NGLLZ,NSPEC_IRREGULAR)
    flattened in Fortran order, select the irregular branch of an element
    (get_gradient_element :603-646 and the fluxes :255-300).  The Fortran
    passes xixstore(:,:,:,ispec) to get_gradient_element and reads
    xixstore(i,j,k,ispec_irreg) for the fluxes; the two are the same row
    when every element is irregular, the case transcribed here.
    """
    import numpy as np
    f32 = np.float32
    N = 5
    nspec = len(dat_in) // 125

    def idx(i, j, k, ispec):               # dat(i,j,k,ispec), all 1-based
        return (i - 1) + N * (j - 1) + 25 * (k - 1) + 125 * (ispec - 1)

    # GLL points, weights, derivative matrices (define_derivation_matrices)
    xigll, wxgll = _gll5()
    hprime_xx = [[f32(0)] * (N + 1) for _ in range(N + 1)]
    hprimewgll_xx = [[f32(0)] * (N + 1) for _ in range(N + 1)]
    for i1 in range(1, N + 1):
        for i2 in range(1, N + 1):
            d = _lagrange_deriv(i1 - 1, i2 - 1, xigll)
            hprime_xx[i2][i1] = f32(d)
            hprimewgll_xx[i2][i1] = f32(wxgll[i2 - 1] * d)
    hprime_xxT = [[f32(0)] * (N + 1) for _ in range(N + 1)]
    for j in range(1, N + 1):
        for i in range(1, N + 1):
            hprime_xxT[j][i] = hprime_xx[i][j]
    wgllwgll = [[f32(wxgll[a - 1] * wxgll[b - 1]) if a and b else f32(0)
                 for b in range(N + 1)] for a in range(N + 1)]

    # rotate_r  (smooth.f90:81-94)
    rot = {}
    if is_sph:
        for ispec in range(1, nspec + 1):
            for k in range(1, N + 1):
                for j in range(1, N + 1):
                    for i in range(1, N + 1):
                        iglob = ibool[idx(i, j, k, ispec)]
                        xl = f32(xstore[iglob - 1])
                        yl = f32(ystore[iglob - 1])
                        zl = f32(zstore[iglob - 1])
                        rl = f32(np.sqrt(f32(f32(xl * xl + yl * yl) + zl * zl)))
                        rot[idx(i, j, k, ispec)] = (f32(xl / rl), f32(yl / rl), f32(zl / rl))

    # cmax, cv, ch, ntstep  (smooth.f90:99-109)
    sh, sv = f32(sigma_h), f32(sigma_v)
    cmax = f32(f32(distance_min_glob) ** 2 / f32(9.0))
    if sv >= sh:
        cv = cmax
        ch = f32(f32(cv * f32(sh ** 2)) / f32(sv ** 2))
    else:
        ch = cmax
        cv = f32(f32(ch * f32(sv ** 2)) / f32(sh ** 2))
    ntstep = int(math.ceil(float(f32(max(sh, sv) ** 2) / f32(2.0 * cmax))))
    if nstep:
        ntstep = nstep

    def irreg_of(ispec):
        return 0 if irregular_element_number is None else int(irregular_element_number[ispec - 1])

    def store(q, i, j, k, row):        # stores[q](i,j,k,row), 1-based
        return f32(stores[q][idx(i, j, k, row)])

    # rvol  (smooth.f90:142-164)
    nglob = max(ibool)
    rvol = [f32(0)] * (nglob + 1)
    rvol_local = [f32(0)] * (125 * nspec)
    for ispec in range(1, nspec + 1):
        for k in range(1, N + 1):
            for j in range(1, N + 1):
                for i in range(1, N + 1):
                    weight = wxgll[i - 1] * wxgll[j - 1] * wxgll[k - 1]
                    ispec_irreg = irreg_of(ispec)
                    if ispec_irreg != 0:
                        jacobianl = store(9, i, j, k, ispec_irreg)
                    else:
                        jacobianl = f32(jacobian_regular)
                    rvol_local[idx(i, j, k, ispec)] = f32(float(jacobianl) * weight)
                    iglob = ibool[idx(i, j, k, ispec)]
                    rvol[iglob] = f32(rvol[iglob] + rvol_local[idx(i, j, k, ispec)])
    for g in range(1, nglob + 1):
        rvol[g] = f32(f32(1.0) / rvol[g])

    dat = [f32(v) for v in dat_in]
    # project  (smooth.f90:193-214)
    dat_glob = [f32(0)] * (nglob + 1)
    for ispec in range(1, nspec + 1):
        for k in range(1, N + 1):
            for j in range(1, N + 1):
                for i in range(1, N + 1):
                    q = idx(i, j, k, ispec)
                    iglob = ibool[q]
                    dat_glob[iglob] = f32(dat_glob[iglob] + f32(dat[q] * rvol_local[q]))
    for g in range(1, nglob + 1):
        dat_glob[g] = f32(dat_glob[g] * rvol[g])
    for q in range(125 * nspec):
        dat[q] = dat_glob[ibool[q]]

    xix = f32(xix_regular)
    for _istep in range(ntstep):                      # smooth.f90:244-370
        ddat_glob = [f32(0)] * (nglob + 1)
        for ispec in range(1, nspec + 1):
            ispec_irreg = irreg_of(ispec)
            dx, dy, dz = {}, {}, {}
            for k in range(1, N + 1):     # get_gradient_element(_regular)
                for j in range(1, N + 1):
                    for i in range(1, N + 1):
                        t1 = t2 = t3 = f32(0)
                        for l in range(1, N + 1):
                            t1 = f32(t1 + f32(dat[idx(l, j, k, ispec)] * hprime_xxT[l][i]))
                        for l in range(1, N + 1):
                            t2 = f32(t2 + f32(dat[idx(i, l, k, ispec)] * hprime_xxT[l][j]))
                        for l in range(1, N + 1):
                            t3 = f32(t3 + f32(dat[idx(i, j, l, ispec)] * hprime_xxT[l][k]))
                        if ispec_irreg != 0:
                            G = [store(q, i, j, k, ispec_irreg) for q in range(9)]
                            dx[(i, j, k)] = f32(f32(f32(t1 * G[0]) + f32(t2 * G[3])) + f32(t3 * G[6]))
                            dy[(i, j, k)] = f32(f32(f32(t1 * G[1]) + f32(t2 * G[4])) + f32(t3 * G[7]))
                            dz[(i, j, k)] = f32(f32(f32(t1 * G[2]) + f32(t2 * G[5])) + f32(t3 * G[8]))
                        else:
                            v = f32(f32(f32(t1 * xix) + f32(t2 * xix)) + f32(t3 * xix))
                            dx[(i, j, k)] = dy[(i, j, k)] = dz[(i, j, k)] = v
            st1, st2, st3 = {}, {}, {}
            jacobianl = f32(jacobian_regular)
            for k in range(1, N + 1):
                for j in range(1, N + 1):
                    for i in range(1, N + 1):
                        a, b, c = dx[(i, j, k)], dy[(i, j, k)], dz[(i, j, k)]
                        if ispec_irreg != 0:
                            G = [store(q, i, j, k, ispec_irreg) for q in range(10)]
                            jl = G[9]
                            sts = []
                            for r in range(3):
                                ax_, ay_, az_ = G[3 * r], G[3 * r + 1], G[3 * r + 2]
                                g = f32(f32(f32(ax_ * a) + f32(ay_ * b)) + f32(az_ * c))
                                if is_sph:
                                    rxl, ryl, rzl = rot[idx(i, j, k, ispec)]
                                    mr = f32(f32(f32(rxl * ax_) + f32(ryl * ay_)) + f32(rzl * az_))
                                    rdot = f32(f32(f32(rxl * a) + f32(ryl * b)) + f32(rzl * c))
                                    v = f32(f32(f32(f32(cv - ch) * mr) * rdot) + f32(ch * g))
                                else:
                                    v = f32(f32(f32(f32(cv - ch) * az_) * c) + f32(ch * g))
                                sts.append(f32(v * jl))
                            st1[(i, j, k)], st2[(i, j, k)], st3[(i, j, k)] = sts
                            continue
                        if is_sph:
                            rxl, ryl, rzl = rot[idx(i, j, k, ispec)]
                            rdot = f32(f32(f32(rxl * a) + f32(ryl * b)) + f32(rzl * c))
                            mr = f32(f32(f32(rxl * xix) + f32(ryl * xix)) + f32(rzl * xix))
                            g = f32(f32(f32(xix * a) + f32(xix * b)) + f32(xix * c))
                            v = f32(f32(f32(f32(cv - ch) * mr) * rdot) + f32(ch * g))
                            v = f32(v * jacobianl)
                        else:
                            g = f32(f32(f32(xix * a) + f32(xix * b)) + f32(xix * c))
                            v = f32(f32(f32(f32(cv - ch) * xix) * c) + f32(ch * g))
                            v = f32(v * jacobianl)
                        st1[(i, j, k)] = st2[(i, j, k)] = st3[(i, j, k)] = v
            for k in range(1, N + 1):
                for j in range(1, N + 1):
                    for i in range(1, N + 1):
                        n1 = n2 = n3 = f32(0)
                        for l in range(1, N + 1):
                            n1 = f32(n1 + f32(st1[(l, j, k)] * hprimewgll_xx[l][i]))
                            n2 = f32(n2 + f32(st2[(i, l, k)] * hprimewgll_xx[l][j]))
                            n3 = f32(n3 + f32(st3[(i, j, l)] * hprimewgll_xx[l][k]))
                        fac1 = wgllwgll[j][k]
                        fac2 = wgllwgll[i][k]
                        fac3 = wgllwgll[i][j]
                        iglob = ibool[idx(i, j, k, ispec)]
                        ddat_glob[iglob] = f32(ddat_glob[iglob] - f32(
                            f32(f32(fac1 * n1) + f32(fac2 * n2)) + f32(fac3 * n3)))
        for g in range(1, nglob + 1):
            ddat_glob[g] = f32(ddat_glob[g] * rvol[g])
            dat_glob[g] = f32(dat_glob[g] + ddat_glob[g])
        if is_cpml is not None:
            for ispec in range(1, nspec + 1):
                if is_cpml[ispec - 1]:
                    for q in range(125 * (ispec - 1), 125 * ispec):
                        dat_glob[ibool[q]] = f32(0)   # dat_bak = 0 (ZERO_PML)
        for q in range(125 * nspec):
            dat[q] = dat_glob[ibool[q]]
    return dat, ntstep


def _gll5():
    """GLL points and weights for 5 points in FP64 (zwgljd)."""
    import numpy as np
    from numpy.polynomial import legendre as L
    c = [0, 0, 0, 0, 1]                            # P_4
    inner = np.sort(np.real(L.legroots(L.legder(c))))
    x = np.concatenate(([-1.0], inner, [1.0]))
    w = 2.0 / (4 * 5 * L.legval(x, c) ** 2)
    return list(x), list(w)


def _lagrange_deriv(i, j, x):
    """Derivative of the i-th Lagrange interpolant at x[j] (0-based)."""
    s = 0.0
    n = len(x)
    for m in range(n):
        if m == i:
            continue
        prod = 1.0 / (x[i] - x[m])
        for q in range(n):
            if q in (i, m):
                continue
            prod *= (x[j] - x[q]) / (x[i] - x[q])
        s += prod
    return s


def xapiir_bu_bp(data, iord, flo, fhi, ts, passes):
    """SAC's XAPIIR for APROTO='BU', TYPE='BP' (src/shared/xapiir_sub.f90:
    58-86 XAPIIR, 118-200 APPLY, 237-304 DESIGN, 334-368 BUROOTS, 712-726
    WARP, 855-961 LPTBP, 1270-1305 BILIN2), REAL/COMPLEX as float32 /
    complex64 like the Fortran.  Returns the filtered trace (float32)."""
    import numpy as np
    f32, c64 = np.float32, np.complex64

    def warp(f, t):
        twopi = f32(6.2831853)
        angle = f32(f32(twopi * f) * t) / f32(2.0)
        w = f32(f32(2.0) * f32(np.tan(angle))) / t
        return f32(w / twopi)

    # BUROOTS
    pi = f32(3.14159265)
    half = iord // 2
    p, rtype = [], []
    if 2 * half < iord:
        p.append(c64(complex(-1.0, 0.0)))
        rtype.append("SP")
    for k in range(1, half + 1):
        angle = f32(pi * f32(f32(0.5) + f32(2 * k - 1) / f32(2 * iord)))
        p.append(c64(complex(np.cos(angle), np.sin(angle))))
        rtype.append("CP")
    dcvalue = f32(1.0)
    # DESIGN: BP mapping
    flw = warp(f32(f32(flo) * f32(ts)) / f32(2.0), f32(2.0))
    fhw = warp(f32(f32(fhi) * f32(ts)) / f32(2.0), f32(2.0))
    # LPTBP
    twopi = f32(f32(2.0) * pi)
    A = f32(f32(f32(twopi * twopi) * flw) * fhw)
    B = f32(twopi * f32(fhw - flw))
    sn, sd = [], []
    for i in range(len(p)):
        if rtype[i] == "CP":
            bp = c64(B * p[i])
            ctemp = c64(np.sqrt(c64(c64(bp * bp) - c64(f32(4.0) * A))))
            p1 = c64(f32(0.5) * c64(bp + ctemp))
            p2 = c64(f32(0.5) * c64(bp - ctemp))
            for q in (p1, p2):
                sn += [f32(0.0), B, f32(0.0)]
                sd += [f32((q * np.conj(q)).real), f32(f32(-2.0) * f32(q.real)), f32(1.0)]
        else:
            sn += [f32(0.0), B, f32(0.0)]
            sd += [A, f32(-B * f32(p[i].real)), f32(1.0)]
    nsects = len(sn) // 3
    s = c64(complex(0.0, float(np.sqrt(A))))
    h = c64(complex(1.0, 0.0))
    for j in range(nsects):
        k = 3 * j
        num = c64(c64(c64(sn[k + 2] * s) + sn[k + 1]) * s) + sn[k]
        den = c64(c64(c64(sd[k + 2] * s) + sd[k + 1]) * s) + sd[k]
        h = c64(h * c64(num / den))
    scale = f32(dcvalue / f32(np.sqrt(f32((h * np.conj(h)).real))))
    sn[0] = f32(sn[0] * scale)
    sn[1] = f32(sn[1] * scale)
    sn[2] = f32(sn[2] * scale)
    # BILIN2
    for j in range(nsects):
        k = 3 * j
        a0, a1, a2 = sd[k], sd[k + 1], sd[k + 2]
        sc = f32(f32(a2 + a1) + a0)
        sd[k] = f32(1.0)
        sd[k + 1] = f32(f32(f32(2.0) * f32(a0 - a2)) / sc)
        sd[k + 2] = f32(f32(f32(a2 - a1) + a0) / sc)
        a0, a1, a2 = sn[k], sn[k + 1], sn[k + 2]
        sn[k] = f32(f32(f32(a2 + a1) + a0) / sc)
        sn[k + 1] = f32(f32(f32(2.0) * f32(a0 - a2)) / sc)
        sn[k + 2] = f32(f32(f32(a2 - a1) + a0) / sc)
    # APPLY
    x = [f32(v) for v in data]
    n = len(x)

    def run(order):
        for j in range(nsects):
            k = 3 * j
            x1 = x2 = y1 = y2 = f32(0.0)
            b0, b1, b2, a1, a2 = sn[k], sn[k + 1], sn[k + 2], sd[k + 1], sd[k + 2]
            for i in order:
                out = f32(f32(f32(b0 * x[i]) + f32(b1 * x1)) + f32(b2 * x2))
                out = f32(out - f32(f32(a1 * y1) + f32(a2 * y2)))
                y2, y1 = y1, out
                x2, x1 = x1, x[i]
                x[i] = out

    run(range(n))
    if passes != 1:
        run(range(n - 1, -1, -1))
    return np.array(x, np.float32)


def detrend(x):
    """src/shared/signal.f90:382-406 line by line (FP64)."""
    n = len(x)
    dan = float(n)
    ds1 = 0.0
    ds2 = 0.0
    for i in range(1, n + 1):
        ds1 = ds1 + x[i - 1]
        ds2 = ds2 + ds1
    davei = 0.5 * (dan + 1.0)
    davex = ds1 / dan
    dslope = -12.0 * (ds2 - davei * ds1) / (dan * (dan * dan - 1.0))
    out = list(x)
    for i in range(1, n + 1):
        dai = float(i - 1)
        out[i - 1] = x[i - 1] - davex - dslope * (dai - davei)
    return out


def interpolate_func_dp(syn, t1, dt1, npt1, t2, dt2, npt2):
    """src/shared/signal.f90:85-125 line by line (FP64)."""
    syn1 = [0.0] * npt2
    for i in range(1, npt2 + 1):
        time = t2 + (i - 1) * dt2
        if time > t1 and time < t1 + (npt1 - 1) * dt1:
            ii = math.floor((time - t1) / dt1) + 1
            tt = time - ((ii - 1) * dt1 + t1)
            syn1[i - 1] = (syn[ii + 1 - 1] - syn[ii - 1]) * tt / dt1 + syn[ii - 1]
    return syn1


def invert_hess(hess):
    """Element by element in FP32, as the Fortran array statements run."""
    import numpy as np
    f = np.float32
    h = [f(x) for x in hess]
    maxh = f(0.0)
    for x in h:
        maxh = max(maxh, f(abs(x)))
    if maxh < f(1.0e-18):
        h = [f(1.0) for _ in h]
    else:
        h = [f(x / maxh) for x in h]
    thr = f(1.0e-3)
    h = [f(f(1.0) / x) if abs(x) > thr else f(f(1.0) / thr) for x in h]
    maxh = f(0.0)
    for x in h:
        maxh = max(maxh, f(abs(x)))
    return [f(x / maxh) for x in h]


def interp1_0(x, v, xq):
    """1-based masked minloc/maxloc as written; returns None where the
    Fortran would read x(0) (xq below the first level)."""
    n = len(x)
    x1 = 0
    best = None
    for i in range(1, n + 1):
        if xq >= x[i - 1] and (best is None or xq - x[i - 1] < best):
            best, x1 = xq - x[i - 1], i
    x2 = 0
    best = None
    for i in range(1, n + 1):
        if xq < x[i - 1] and (best is None or xq - x[i - 1] > best):
            best, x2 = xq - x[i - 1], i
    if x2 != 0:
        if x1 == 0:
            return None
        vn = abs(x[x2 - 1] - x[x1 - 1])
        vq = v[x1 - 1] * (x[x2 - 1] - xq) + v[x2 - 1] * (xq - x[x1 - 1])
        return vq / vn
    if xq <= x[0]:
        return v[0]
    if xq >= x[n - 1]:
        return v[n - 1]
    return None


def get_1d_precond(zgrid, precond_type):
    import numpy as np
    f = np.float32
    zl = []
    for z in zgrid:
        if f(z) > f(0.0):
            q = f(1.0e-8)
        else:
            q = f(f(z) + f(1.0e-8))
        if precond_type == 2:
            q = f(f(1.0) / f(np.sqrt(f(q * q))))
        elif precond_type == 3:
            q = f(f(1.0) / f(np.sqrt(f(np.sqrt(f(q * q))))))
        zl.append(q)
    return zl


def zprecond_gll(ibool, zstore, zgrid, precond_type, nevents):
    """ibool: flat 1-based element-point -> global point; returns the flat
    FP32 preconditioner."""
    import numpy as np
    f = np.float32
    zl = [float(q) for q in get_1d_precond(zgrid, precond_type)]
    zg = [float(z) for z in zgrid]
    h = [f(interp1_0(zg, zl, float(zstore[ig - 1]))) for ig in ibool]
    h = [f(x * f(nevents)) for x in h]
    maxh = max(f(abs(x)) for x in h)
    h = [f(x / maxh) for x in h]
    h = [f(f(1.0) / x) for x in h]
    maxh = max(f(abs(x)) for x in h)
    return [f(x / maxh) for x in h]


def coswin(n, opt):
    import numpy as np
    f = np.float32
    nn = 2 * n + 1
    win = [f(0.5) - f(0.5) * f(np.cos(f(2.0) * f(3.1415926535) * f(i - 1) / f(nn - 1)))
           for i in range(1, nn + 1)]
    return win[0:n] if opt == 1 else win[n + 1:nn]


def create_taper(taph1, taph2, tapz1, tapz2, hx, hy, hz, nx, ny, nz):
    import numpy as np
    f = np.float32
    xt = [f(0.0)] * (nx + 1)
    yt = [f(0.0)] * (ny + 1)
    zt = [f(0.0)] * (nz + 1)
    nh1 = int(np.floor(f(taph1) / f(hx)))
    nh2 = int(np.floor(f(taph2) / f(hx)))
    x1, x2, x3, x4 = nh1 + 1, nh1 + nh2 + 1, nx - nh1 - nh2, nx - nh1
    for q, v in zip(range(x1, x2), coswin(nh2, 1)):
        xt[q] = v
    for q, v in zip(range(x3 + 1, x4 + 1), coswin(nh2, 0)):
        xt[q] = v
    for q in range(x2, x3 + 1):
        xt[q] = f(1.0)
    nh1 = int(np.floor(f(taph1) / f(hy)))
    nh2 = int(np.floor(f(taph2) / f(hy)))
    y1, y2, y3, y4 = nh1 + 1, nh1 + nh2 + 1, ny - nh1 - nh2, ny - nh1
    for q, v in zip(range(y1, y2), coswin(nh2, 1)):
        yt[q] = v
    for q, v in zip(range(y3 + 1, y4 + 1), coswin(nh2, 0)):
        yt[q] = v
    for q in range(y2, y3 + 1):
        yt[q] = f(1.0)
    nh1 = int(np.floor(f(tapz1) / f(hz)))
    nh2 = int(np.floor(f(tapz2) / f(hz)))
    z1 = nh1 + nh2 + 1
    for q, v in zip(range(nh1 + 1, z1), coswin(nh2, 1)):
        zt[q] = v
    for q in range(z1, nz + 1):
        zt[q] = f(1.0)
    out = np.zeros((nx, ny, nz), np.float32)
    for k in range(1, nz + 1):
        for j in range(1, ny + 1):
            for i in range(1, nx + 1):
                out[i - 1, j - 1, k - 1] = xt[i] * yt[j] * zt[k]
    return out


def locate_bissection(valx, n, x):
    if x < valx[0] or x > valx[n - 1]:
        return -1
    jl, ju = 0, n + 1
    while ju - jl > 1:
        jm = (ju + jl) // 2
        if x >= valx[jm - 1]:
            jl = jm
        else:
            ju = jm
    if x == valx[0]:
        return 1
    if x == valx[n - 1]:
        return n - 1
    return jl


def interp3(valx, valy, valz, valin, x, y, z):
    nx, ny, nz = len(valx), len(valy), len(valz)
    indx = locate_bissection(valx, nx, x)
    indy = locate_bissection(valy, ny, y)
    indz = locate_bissection(valz, nz, z)
    kx = min(max(indx, 1), nx - 1)
    ky = min(max(indy, 1), ny - 1)
    kz = min(max(indz, 1), nz - 1)
    X = lambda q: valx[q - 1]  # noqa: E731
    Y = lambda q: valy[q - 1]  # noqa: E731
    Z = lambda q: valz[q - 1]  # noqa: E731
    V = lambda a, b, c: valin[a - 1][b - 1][c - 1]  # noqa: E731
    xix1, yiy1, ziz1 = x - X(kx), y - Y(ky), z - Z(kz)
    xix2, yiy2, ziz2 = x - X(kx + 1), y - Y(ky + 1), z - Z(kz + 1)
    x1x2, y1y2, z1z2 = 1.0 / (X(kx) - X(kx + 1)), 1.0 / (Y(ky) - Y(ky + 1)), 1.0 / (Z(kz) - Z(kz + 1))
    x2x1, y2y1, z2z1 = 1.0 / (X(kx + 1) - X(kx)), 1.0 / (Y(ky + 1) - Y(ky)), 1.0 / (Z(kz + 1) - Z(kz))
    return (xix2 * yiy2 * ziz2 * x1x2 * y1y2 * z1z2 * V(kx, ky, kz)
            + xix2 * yiy2 * ziz1 * x1x2 * y1y2 * z2z1 * V(kx, ky, kz + 1)
            + xix2 * yiy1 * ziz2 * x1x2 * y2y1 * z1z2 * V(kx, ky + 1, kz)
            + xix2 * yiy1 * ziz1 * x1x2 * y2y1 * z2z1 * V(kx, ky + 1, kz + 1)
            + xix1 * yiy2 * ziz2 * x2x1 * y1y2 * z1z2 * V(kx + 1, ky, kz)
            + xix1 * yiy2 * ziz1 * x2x1 * y1y2 * z2z1 * V(kx + 1, ky, kz + 1)
            + xix1 * yiy1 * ziz2 * x2x1 * y2y1 * z1z2 * V(kx + 1, ky + 1, kz)
            + xix1 * yiy1 * ziz1 * x2x1 * y2y1 * z2z1 * V(kx + 1, ky + 1, kz + 1))


def get_nearest_bound_idx(x, x_sem):
    n = len(x)
    indx = None   # left undefined by the Fortran for a point inside the axis
    if x_sem < x[0]:
        indx = 1
    elif x_sem > x[n - 1]:
        indx = n - 1
    return indx


def interp3_nearest_simple(x, y, z, model, x_sem, y_sem, z_sem):
    nx, ny, nz = len(x), len(y), len(z)
    min_dist = 1.0e30
    value = None
    indx = locate_bissection(x, nx, x_sem)
    indy = locate_bissection(y, ny, y_sem)
    indz = locate_bissection(z, nz, z_sem)
    m = 2
    if indx != -1:
        kx = min(max(indx - (m - 1) // 2, 1), nx + 1 - m)
    else:
        kx = get_nearest_bound_idx(x, x_sem)
    if indy != -1:
        ky = min(max(indy - (m - 1) // 2, 1), ny + 1 - m)
    else:
        ky = get_nearest_bound_idx(y, y_sem)
    if indz != -1:
        kz = min(max(indz - (m - 1) // 2, 1), nz + 1 - m)
    else:
        kz = get_nearest_bound_idx(z, z_sem)
    for ifd in range(kx, kx + 1 + 1):
        xfd = x[ifd - 1]
        for jfd in range(ky, ky + 1 + 1):
            yfd = y[jfd - 1]
            for kfd in range(kz, kz + 1 + 1):
                zfd = z[kfd - 1]
                dist = math.sqrt((x_sem - xfd) ** 2 + (y_sem - yfd) ** 2 + (z_sem - zfd) ** 2)
                if dist < min_dist and model[ifd - 1][jfd - 1][kfd - 1] != 0.0:
                    min_dist = dist
                    value = model[ifd - 1][jfd - 1][kfd - 1]
    return value


def model_external_values(x, y, z, vp, vs, rho, xsem, ysem, zsem):
    """vp, vs, rho at one GLL point (model_external_values.f90:206-273)."""
    if (xsem < x[0] or xsem > x[len(x) - 1] or ysem < y[0] or ysem > y[len(y) - 1]
            or zsem < z[0] or zsem > z[len(z) - 1]):
        r = interp3_nearest_simple(x, y, z, rho, xsem, ysem, zsem)
        p = interp3_nearest_simple(x, y, z, vp, xsem, ysem, zsem)
        s = interp3_nearest_simple(x, y, z, vs, xsem, ysem, zsem)
    else:
        r = interp3(x, y, z, rho, xsem, ysem, zsem)
        p = interp3(x, y, z, vp, xsem, ysem, zsem)
        s = interp3(x, y, z, vs, xsem, ysem, zsem)
    return p, s, r


def project_sem2fd(ibool, xstore, ystore, zstore, nspec, data, ox, oy, oz, hx, hy, hz,
                   nx, ny, nz):
    """ibool: flat 1-based (i fastest); data: flat element values in the
    same order.  Returns the grid as nested lists [nx][ny][nz]."""
    import math
    xg = [-1.0, -math.sqrt(3.0 / 7.0), 0.0, math.sqrt(3.0 / 7.0), 1.0]

    def lag(x):
        out = []
        for i in range(5):
            v = 1.0
            for m in range(5):
                if m != i:
                    v *= (x - xg[m]) / (xg[i] - xg[m])
            out.append(v)
        return out
    found = {}
    for ispec in range(1, nspec + 1):
        xs = [xstore[ibool[(ispec - 1) * 125 + q] - 1] for q in range(125)]
        ys = [ystore[ibool[(ispec - 1) * 125 + q] - 1] for q in range(125)]
        zs = [zstore[ibool[(ispec - 1) * 125 + q] - 1] for q in range(125)]
        xmin, xmax, ymin, ymax = min(xs), max(xs), min(ys), max(ys)
        zmin, zmax = min(zs), max(zs)
        kmin, kmax = int(1 + (zmin - oz) / hz), int(1 + (zmax - oz) / hz)
        jmin, jmax = int(1 + (ymin - oy) / hy), int(1 + (ymax - oy) / hy)
        imin, imax = int(1 + (xmin - ox) / hx), int(1 + (xmax - ox) / hx)
        for kfd in range(kmin, kmax + 1):
            zfd = oz + (kfd - 1) * hz
            for jfd in range(jmin, jmax + 1):
                yfd = oy + (jfd - 1) * hy
                for ifd in range(imin, imax + 1):
                    xfd = ox + (ifd - 1) * hx
                    if not (1 <= ifd <= nx and 1 <= jfd <= ny and 1 <= kfd <= nz):
                        continue
                    # locate_point_in_element: Newton steps (exact for
                    # these affine elements), each clamped to [-1, 1]
                    xi = min(max(2.0 * (xfd - xmin) / (xmax - xmin) - 1.0, -1.0), 1.0)
                    eta = min(max(2.0 * (yfd - ymin) / (ymax - ymin) - 1.0, -1.0), 1.0)
                    gam = min(max(2.0 * (zfd - zmin) / (zmax - zmin) - 1.0, -1.0), 1.0)
                    if abs(xi) < 1.05 and abs(eta) < 1.05 and abs(gam) < 1.05:
                        if (ifd, jfd, kfd) not in found:
                            found[(ifd, jfd, kfd)] = (ispec, xi, eta, gam)
    grid = [[[0.0] * nz for _ in range(ny)] for _ in range(nx)]
    for (ifd, jfd, kfd), (ispec, xi, eta, gam) in found.items():
        hxis, hetas, hgams = lag(xi), lag(eta), lag(gam)
        val = 0.0
        for kgg in range(5):
            for jgg in range(5):
                for igg in range(5):
                    val += hxis[igg] * hetas[jgg] * hgams[kgg] * \
                        data[(ispec - 1) * 125 + igg + 5 * jgg + 25 * kgg]
        grid[ifd - 1][jfd - 1][kfd - 1] = val
    return grid


def _inv3(m):
    a, b, c = m[0]
    d, e, f = m[1]
    g, h, i = m[2]
    det = a * (e * i - f * h) - b * (d * i - f * g) + c * (d * h - e * g)
    return [[(e * i - f * h) / det, (c * h - b * i) / det, (b * f - c * e) / det],
            [(f * g - d * i) / det, (a * i - c * g) / det, (c * d - a * f) / det],
            [(d * h - e * g) / det, (b * g - a * h) / det, (a * e - b * d) / det]]


def locate_point_in_element(ex, ey, ez, xt, yt, zt, niter=4):
    """ex, ey, ez: the element's 125 GLL point coordinates, i fastest."""
    import math
    xg = [-1.0, -math.sqrt(3.0 / 7.0), 0.0, math.sqrt(3.0 / 7.0), 1.0]
    P = lambda i, j, k: (i - 1) + 5 * (j - 1) + 25 * (k - 1)  # noqa: E731
    distmin = float("inf")
    ig = jg = kg = 1
    for k in range(2, 5):
        for j in range(2, 5):
            for i in range(2, 5):
                q = P(i, j, k)
                dist = (xt - ex[q]) ** 2 + (yt - ey[q]) ** 2 + (zt - ez[q]) ** 2
                if dist < distmin:
                    distmin, ig, jg, kg = dist, i, j, k
    xi, eta, gam = xg[ig - 1], xg[jg - 1], xg[kg - 1]
    corners = [(a, b, c) for c in (0, 1) for b in (0, 1) for a in (0, 1)]
    anc = [P(1 + 4 * a, 1 + 4 * b, 1 + 4 * c) for (a, b, c) in corners]
    for _ in range(niter):
        x = y = z = 0.0
        J = [[0.0] * 3 for _ in range(3)]
        for (a, b, c), q in zip(corners, anc):
            sa, sb, sc = (1 - 2 * a), (1 - 2 * b), (1 - 2 * c)
            la = 0.5 * (1 - sa * xi)
            lb = 0.5 * (1 - sb * eta)
            lc = 0.5 * (1 - sc * gam)
            dla, dlb, dlc = -0.5 * sa, -0.5 * sb, -0.5 * sc
            n = la * lb * lc
            dn = (dla * lb * lc, la * dlb * lc, la * lb * dlc)
            x += n * ex[q]
            y += n * ey[q]
            z += n * ez[q]
            for e_ in range(3):
                J[0][e_] += dn[e_] * ex[q]
                J[1][e_] += dn[e_] * ey[q]
                J[2][e_] += dn[e_] * ez[q]
        inv = _inv3(J)
        dx, dy, dz = -(x - xt), -(y - yt), -(z - zt)
        xi += inv[0][0] * dx + inv[0][1] * dy + inv[0][2] * dz
        eta += inv[1][0] * dx + inv[1][1] * dy + inv[1][2] * dz
        gam += inv[2][0] * dx + inv[2][1] * dy + inv[2][2] * dz
        xi, eta, gam = (min(max(v, -1.0), 1.0) for v in (xi, eta, gam))
    return xi, eta, gam


def project_sem2fd_located(ibool, xstore, ystore, zstore, nspec, data, ox, oy, oz, hx, hy,
                           hz, nx, ny, nz):
    """As project_sem2fd, with locate_point_in_element for every element."""
    import math
    xg = [-1.0, -math.sqrt(3.0 / 7.0), 0.0, math.sqrt(3.0 / 7.0), 1.0]

    def lag(x):
        out = []
        for i in range(5):
            v = 1.0
            for m in range(5):
                if m != i:
                    v *= (x - xg[m]) / (xg[i] - xg[m])
            out.append(v)
        return out
    found = {}
    for ispec in range(1, nspec + 1):
        ex = [xstore[ibool[(ispec - 1) * 125 + q] - 1] for q in range(125)]
        ey = [ystore[ibool[(ispec - 1) * 125 + q] - 1] for q in range(125)]
        ez = [zstore[ibool[(ispec - 1) * 125 + q] - 1] for q in range(125)]
        kmin, kmax = int(1 + (min(ez) - oz) / hz), int(1 + (max(ez) - oz) / hz)
        jmin, jmax = int(1 + (min(ey) - oy) / hy), int(1 + (max(ey) - oy) / hy)
        imin, imax = int(1 + (min(ex) - ox) / hx), int(1 + (max(ex) - ox) / hx)
        for kfd in range(kmin, kmax + 1):
            for jfd in range(jmin, jmax + 1):
                for ifd in range(imin, imax + 1):
                    if not (1 <= ifd <= nx and 1 <= jfd <= ny and 1 <= kfd <= nz):
                        continue
                    if (ifd, jfd, kfd) in found:
                        continue
                    loc = locate_point_in_element(ex, ey, ez, ox + (ifd - 1) * hx,
                                                  oy + (jfd - 1) * hy, oz + (kfd - 1) * hz)
                    if all(abs(v) < 1.05 for v in loc):
                        found[(ifd, jfd, kfd)] = (ispec,) + tuple(loc)
    grid = [[[0.0] * nz for _ in range(ny)] for _ in range(nx)]
    for (ifd, jfd, kfd), (ispec, xi, eta, gam) in found.items():
        hxis, hetas, hgams = lag(xi), lag(eta), lag(gam)
        val = 0.0
        for kgg in range(5):
            for jgg in range(5):
                for igg in range(5):
                    val += hxis[igg] * hetas[jgg] * hgams[kgg] * \
                        data[(ispec - 1) * 125 + igg + 5 * jgg + 25 * kgg]
        grid[ifd - 1][jfd - 1][kfd - 1] = val
    return grid
