"""File formats at either side of the solver, as the reference writes them.

Inputs:
- ``read_cmtsolution``: CMTSOLUTION files, which the reference reads with
  SPECFEM's ``get_cmt`` (called at src/specfem_interface/
  locate_source_fwat.f90:890).  Moment tensor in dyne-cm, depth in km.
- ``read_stations``: STATIONS lines "name network lat lon elevation
  burial".
- ``read_sac``: SAC binary traces, the observed data (src/shared/sacio.f90).

Outputs:
- ``write_adj_ascii`` and ``read_adj_ascii``: SEM/<net>.<sta>.<comp>.adj
  adjoint sources, two columns "time value" (``dwascii``,
  src/shared/common.f90:226-244, written by ``write_adj``,
  src/preproc/syn_data.f90:232-251).
- ``write_kernel_bin`` and ``read_kernel_bin``: procNNNNNN_<name>.bin
  element arrays dat(NGLLX,NGLLY,NGLLZ,NSPEC), one Fortran unformatted
  sequential record of float32 (4-byte length, payload, 4-byte length).
  The reference reads them in src/postproc/kernel_io.f90:79-98 and names
  the kernels in src/postproc/post_processing.f90:417-422.
- ``write_sac``.
"""
from __future__ import annotations

import os
import struct

import numpy as np

KERNEL_NAMES = ("rho", "mu", "kappa", "rhop", "beta", "alpha")


# -- Fortran unformatted records ------------------------------------------------

def write_kernel_bin(path, data):
    """One record of float32 values in Fortran order. ``data`` is
    [nspec, 5, 5, 5] in this package's layout (index i fastest), which is
    the same memory order as dat(i,j,k,ispec)."""
    a = np.ascontiguousarray(data, np.float32).reshape(-1)
    n = a.nbytes
    with open(path, "wb") as f:
        f.write(struct.pack("<i", n))
        f.write(a.tobytes())
        f.write(struct.pack("<i", n))


def read_kernel_bin(path, nspec=None):
    """Read one record of float32 element values; returns [nspec, 5, 5, 5].
    Raises ValueError when the record markers or the size do not match."""
    with open(path, "rb") as f:
        raw = f.read()
    if len(raw) < 8:
        raise ValueError(f"{path}: too short for a Fortran record")
    (n,) = struct.unpack("<i", raw[:4])
    if n < 0 or len(raw) != n + 8 or struct.unpack("<i", raw[4 + n:8 + n])[0] != n:
        raise ValueError(f"{path}: not one Fortran unformatted record")
    if n % (4 * 125):
        raise ValueError(f"{path}: {n} bytes is not a whole number of elements")
    a = np.frombuffer(raw[4:4 + n], dtype="<f4").astype(np.float32)
    ns = n // (4 * 125)
    if nspec is not None and ns != nspec:
        raise ValueError(f"{path}: {ns} elements, expected {nspec}")
    return a.reshape(ns, 5, 5, 5)


def write_event_kernels(directory, rank, kernels, names=KERNEL_NAMES):
    """procNNNNNN_<name>_kernel.bin for each of the six kernels
    ([6, nspec, 5, 5, 5], the order sem_save_adjoint_kernels returns)."""
    os.makedirs(directory, exist_ok=True)
    paths = []
    for name, k in zip(names, kernels):
        p = os.path.join(directory, f"proc{rank:06d}_{name}_kernel.bin")
        write_kernel_bin(p, k)
        paths.append(p)
    return paths


# -- adjoint sources -------------------------------------------------------------

def write_adj_ascii(path, data, t0, dt):
    """Two columns, b + dt*(i-1) and the value, one line per sample, with
    b = -t0 as write_adj passes it."""
    d = np.asarray(data, np.float64)
    t = -t0 + dt * np.arange(d.size)
    with open(path, "w") as f:
        for ti, v in zip(t, d):
            f.write(f" {ti:25.16E} {v:25.16E}\n")


def read_adj_ascii(path):
    """Returns (times, values) of a two-column ASCII trace."""
    a = np.loadtxt(path, dtype=np.float64, ndmin=2)
    return a[:, 0], a[:, 1]


def write_adjoint_sources(directory, stations, adj, t0, dt, comp_names=("BXE", "BXN", "BXZ")):
    """SEM/<net>.<sta>.<comp>.adj for adj [nrec, 3, nstep] (x=E, y=N, z=Z);
    ``stations`` as read_stations returns them."""
    os.makedirs(directory, exist_ok=True)
    for r, st in enumerate(stations):
        for c in range(3):
            write_adj_ascii(os.path.join(directory, f"{st['network']}.{st['name']}."
                                                    f"{comp_names[c]}.adj"),
                            adj[r, c], t0, dt)


# -- source and station files ----------------------------------------------------

def read_cmtsolution(path):
    """CMTSOLUTION: a header line, then "key: value" lines.  Returns a dict
    with name, time_shift, hdur, lat (or UTM y), lon (or UTM x), depth (km)
    and mt = (Mrr, Mtt, Mpp, Mrt, Mrp, Mtp) in dyne-cm."""
    with open(path) as f:
        lines = [ln.rstrip("\n") for ln in f if ln.strip()]
    vals = {}
    for ln in lines[1:]:
        if ":" not in ln:
            continue
        k, v = ln.split(":", 1)
        vals[k.strip().lower()] = v.strip()

    def num(key):
        return float(vals[key].replace("d", "e").replace("D", "e"))
    return {
        "header": lines[0].strip(),
        "name": vals.get("event name", ""),
        "time_shift": num("time shift"),
        "hdur": num("half duration"),
        "lat": num("latorutm"),
        "lon": num("longorutm"),
        "depth": num("depth"),
        "mt": tuple(num(k) for k in ("mrr", "mtt", "mpp", "mrt", "mrp", "mtp")),
    }


def cmt_to_source(cmt, length_unit=1000.0, ricker=True):
    """Source arguments (x, y, z, mt in N m, f0, tshift) for
    ``solver.make_source`` on a Cartesian mesh (UTM projection suppressed):
    x = longorUTM, y = latorUTM, z = -depth * length_unit (depth in km);
    the moment tensor converts from dyne-cm to N m (1e-7).  With the Ricker
    time function the "half duration" line holds f0 (locate_source_fwat.f90:
    499-506)."""
    if not ricker:
        raise NotImplementedError("only the Ricker source time function is implemented")
    mt = tuple(m * 1e-7 for m in cmt["mt"])
    return (cmt["lon"], cmt["lat"], -cmt["depth"] * length_unit, mt, cmt["hdur"],
            cmt["time_shift"])


def read_stations(path):
    """STATIONS: name network lat(or y) lon(or x) elevation burial."""
    out = []
    with open(path) as f:
        for ln in f:
            p = ln.split()
            if len(p) < 6:
                continue
            out.append({"name": p[0], "network": p[1], "lat": float(p[2]),
                        "lon": float(p[3]), "elevation": float(p[4]),
                        "burial": float(p[5])})
    return out


def stations_xyz(stations, z_surface=0.0):
    """Receiver coordinates on a Cartesian mesh: x = lon, y = lat,
    z = z_surface - burial."""
    return np.array([[s["lon"], s["lat"], z_surface - s["burial"]] for s in stations],
                    np.float64)


# -- SAC binary -----------------------------------------------------------------
# Header: 70 float32, 40 int32, 192 bytes of text; then npts float32.
_F = {"delta": 0, "depmin": 1, "depmax": 2, "b": 5, "e": 6, "o": 7, "a": 8,
      "stla": 31, "stlo": 32, "stel": 33, "stdp": 34, "evla": 35, "evlo": 36,
      "evel": 37, "evdp": 38, "mag": 39, "dist": 50, "az": 51, "baz": 52,
      "gcarc": 53, "depmen": 56, "cmpaz": 57, "cmpinc": 58}
_I = {"nzyear": 0, "nzjday": 1, "nzhour": 2, "nzmin": 3, "nzsec": 4, "nzmsec": 5,
      "nvhdr": 6, "npts": 9, "iftype": 15, "idep": 16, "iztype": 17, "leven": 35}
_UNDEF = -12345.0


def read_sac(path):
    """Returns (header dict, data float32).  Detects byte order from nvhdr."""
    with open(path, "rb") as f:
        raw = f.read()
    if len(raw) < 632:
        raise ValueError(f"{path}: shorter than a SAC header")
    for bo in ("<", ">"):
        ints = np.frombuffer(raw[280:440], dtype=bo + "i4")
        if ints[6] == 6:
            break
    else:
        raise ValueError(f"{path}: not a SAC file (nvhdr != 6)")
    fl = np.frombuffer(raw[:280], dtype=bo + "f4")
    hdr = {k: float(fl[i]) for k, i in _F.items()}
    hdr.update({k: int(ints[i]) for k, i in _I.items()})
    hdr["kstnm"] = raw[440:448].decode("ascii", "replace").strip()
    hdr["kcmpnm"] = raw[440 + 8 * 20:440 + 8 * 21].decode("ascii", "replace").strip()
    hdr["knetwk"] = raw[440 + 8 * 21:440 + 8 * 22].decode("ascii", "replace").strip()
    n = hdr["npts"]
    if len(raw) < 632 + 4 * n:
        raise ValueError(f"{path}: {n} samples announced, file too short")
    data = np.frombuffer(raw[632:632 + 4 * n], dtype=bo + "f4").astype(np.float32)
    return hdr, data


def write_sac(path, data, delta, b=0.0, **fields):
    """Evenly sampled little-endian SAC file (nvhdr 6, iftype time series,
    leven true), with any float/int header fields of _F/_I given by name."""
    d = np.ascontiguousarray(data, np.float32)
    fl = np.full(70, _UNDEF, np.float32)
    ints = np.full(40, -12345, np.int32)
    fl[_F["delta"]], fl[_F["b"]] = delta, b
    fl[_F["e"]] = b + delta * (d.size - 1)
    fl[_F["depmin"]], fl[_F["depmax"]] = float(d.min()), float(d.max())
    fl[_F["depmen"]] = float(d.mean())
    ints[_I["nvhdr"]], ints[_I["npts"]] = 6, d.size
    ints[_I["iftype"]], ints[_I["leven"]] = 1, 1
    for k, v in fields.items():
        if k in _F:
            fl[_F[k]] = v
        elif k in _I:
            ints[_I[k]] = v
        else:
            raise KeyError(k)
    txt = bytearray(b"-12345  " * 24)
    with open(path, "wb") as f:
        f.write(fl.astype("<f4").tobytes())
        f.write(ints.astype("<i4").tobytes())
        f.write(bytes(txt))
        f.write(d.astype("<f4").tobytes())
