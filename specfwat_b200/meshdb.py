"""``proc*_external_mesh.bin``: the mesh database the reference solver reads.

``read_mesh_databases_fwat`` (src/specfem_interface/read_mesh_databases.f90:
91-1200) reads one Fortran unformatted sequential file per slice, written
by SPECFEM's database generator (absent from the tree).  Every array is one
record (4-byte little-endian length, payload, 4-byte length); integers,
reals (CUSTOM_REAL = 4 bytes) and logicals are 4 bytes.  Which records are
present depends on the mesh (acoustic / elastic / poroelastic elements, the
``ispec_is_*`` records) and on Par_file switches (APPROXIMATE_OCEAN_LOAD,
PML_CONDITIONS, STACEY_ABSORBING_CONDITIONS, ANISOTROPY); those are
arguments here.  Three check words (9999, 9998, 9997, 9996) are verified
where the reference verifies them.

``read_external_mesh`` walks the records in the reference's order and
returns them by the reference's names; ``to_database`` turns an elastic
slice into the :class:`~specfwat_b200.database.Database` the solver takes
(``Mesh(db)``; indices made 0-based).  ``write_external_mesh`` writes an
elastic slice in the same order (single slice, no PML, no MPI interfaces),
for converting the synthetic boxes and for the round-trip tests; the
reader is pinned by that order, since no database file from the reference
generator is available here.
"""
from __future__ import annotations

import struct

import numpy as np

from .database import Database

NGLL3 = 125


class _Records:
    """Sequential reader of Fortran unformatted records."""

    def __init__(self, path):
        self.f = open(path, "rb")
        self.path = path

    def close(self):
        self.f.close()

    def raw(self):
        head = self.f.read(4)
        if len(head) < 4:
            raise ValueError(f"{self.path}: unexpected end of file")
        (n,) = struct.unpack("<i", head)
        body = self.f.read(n)
        tail = self.f.read(4)
        if len(body) != n or len(tail) < 4 or struct.unpack("<i", tail)[0] != n:
            raise ValueError(f"{self.path}: broken record markers")
        return body

    def i4(self):
        return np.frombuffer(self.raw(), "<i4")

    def f4(self):
        return np.frombuffer(self.raw(), "<f4")

    def int(self):
        a = self.i4()
        if a.size != 1:
            raise ValueError(f"{self.path}: expected one integer, got {a.size}")
        return int(a[0])

    def logical(self):
        return self.i4() != 0

    def check(self, word):
        w = self.int()
        if w != word:
            raise ValueError(f"{self.path}: database check word {w} where {word} was expected")


def read_external_mesh(path, *, ocean_load=False, pml=False, stacey=True, anisotropy=False):
    """Records of one ``proc*_external_mesh.bin``, by the reference's names.

    Follows read_mesh_databases.f90:158-1146 up to the inner/outer element
    lists; arrays are flat (Fortran order) except the counts."""
    r = _Records(path)
    d = {}

    def sized(name, arr, n, hint=""):
        if arr.size != n:
            raise ValueError(f"{path}: record {name} holds {arr.size} values, {n} expected"
                             + (f" ({hint})" if hint else ""))
        return arr

    try:
        # :158-189
        d["NSPEC_AB"] = r.int()
        d["NGLOB_AB"] = r.int()
        d["NSPEC_IRREGULAR"] = r.int()
        ne = d["NSPEC_AB"] * NGLL3
        d["ibool"] = sized("ibool", r.i4(), ne)
        for k in ("xstore", "ystore", "zstore"):
            d[k] = sized(k, r.f4(), d["NGLOB_AB"])
        d["irregular_element_number"] = r.i4()
        d["xix_regular"] = float(r.f4()[0])
        d["jacobian_regular"] = float(r.f4()[0])
        for k in ("xixstore", "xiystore", "xizstore", "etaxstore", "etaystore", "etazstore",
                  "gammaxstore", "gammaystore", "gammazstore", "jacobianstore"):
            d[k] = r.f4()
        for k in ("kappastore", "mustore", "rhostore"):
            d[k] = r.f4()
        for k in ("ispec_is_acoustic", "ispec_is_elastic", "ispec_is_poroelastic"):
            d[k] = r.logical()
        r.check(9999)
        acoustic = bool(d["ispec_is_acoustic"].any())
        elastic = bool(d["ispec_is_elastic"].any())
        poro = bool(d["ispec_is_poroelastic"].any())
        # :250-494
        if acoustic:
            d["rmass_acoustic"] = r.f4()
        if elastic:
            d["rmass"] = r.f4()
            if ocean_load:
                d["rmass_ocean_load"] = r.f4()
            d["rho_vp"] = r.f4()
            d["rho_vs"] = r.f4()
        # :497-632
        if poro:
            for k in ("rmass_solid_poroelastic", "rmass_fluid_poroelastic", "rhoarraystore",
                      "kappaarraystore", "etastore", "tortstore", "permstore", "phistore",
                      "rho_vpI", "rho_vpII", "rho_vsI"):
                d[k] = r.f4()
        # :652-763
        if pml:
            d["NSPEC_CPML"] = r.int()
            for k in ("CPML_width_x", "CPML_width_y", "CPML_width_z",
                      "min_distance_between_CPML_parameter"):
                d[k] = float(r.f4()[0])
            if d["NSPEC_CPML"] > 0:
                d["CPML_regions"] = r.i4()
                d["CPML_to_spec"] = r.i4()
                d["is_CPML"] = r.logical()
                for k in ("d_store_x", "d_store_y", "d_store_z", "k_store_x", "k_store_y",
                          "k_store_z", "alpha_store_x", "alpha_store_y", "alpha_store_z"):
                    d[k] = r.f4()
                d["nglob_interface_PML_acoustic"] = r.int()
                d["nglob_interface_PML_elastic"] = r.int()
                if d["nglob_interface_PML_acoustic"] > 0:
                    d["points_interface_PML_acoustic"] = r.i4()
                if d["nglob_interface_PML_elastic"] > 0:
                    d["points_interface_PML_elastic"] = r.i4()
        # :766-821
        nf = d["num_abs_boundary_faces"] = r.int()
        if nf < 0:
            raise ValueError(f"{path}: num_abs_boundary_faces < 0")
        if nf > 0:
            d["abs_boundary_ispec"] = r.i4()
            d["abs_boundary_ijk"] = r.i4()
            d["abs_boundary_jacobian2Dw"] = r.f4()
            d["abs_boundary_normal"] = r.f4()
            if stacey and not pml:
                if elastic:
                    for k in ("rmassx", "rmassy", "rmassz"):
                        d[k] = r.f4()
                if acoustic:
                    d["rmassz_acoustic"] = r.f4()
        r.check(9998)
        # :824-869
        names2d = ("nspec2D_xmin", "nspec2D_xmax", "nspec2D_ymin", "nspec2D_ymax",
                   "NSPEC2D_BOTTOM", "NSPEC2D_TOP")
        for k in names2d:
            d[k] = r.int()
        for k, b in zip(names2d, ("ibelm_xmin", "ibelm_xmax", "ibelm_ymin", "ibelm_ymax",
                                  "ibelm_bottom", "ibelm_top")):
            if d[k] > 0:
                d[b] = r.i4()
        # :872-994
        for tag, arrays in (("free_surface", ("ispec", "ijk", "jacobian2Dw", "normal")),
                            ("coupling_ac_el", ("ispec", "ijk", "jacobian2Dw", "normal")),
                            ("coupling_ac_po", ("ispec", "ijk", "jacobian2Dw", "normal"))):
            n = d[f"num_{tag}_faces"] = r.int()
            if n > 0:
                for a in arrays:
                    d[f"{tag}_{a}"] = r.f4() if a in ("jacobian2Dw", "normal") else r.i4()
        n = d["num_coupling_el_po_faces"] = r.int()
        if n > 0:
            d["coupling_el_po_ispec"] = r.i4()
            d["coupling_po_el_ispec"] = r.i4()
            d["coupling_el_po_ijk"] = r.i4()
            d["coupling_po_el_ijk"] = r.i4()
            d["coupling_el_po_jacobian2Dw"] = r.f4()
            d["coupling_el_po_normal"] = r.f4()
        r.check(9997)
        # :1003-1047
        d["num_interfaces_ext_mesh"] = r.int()
        d["max_nibool_interfaces_ext_mesh"] = r.int()
        if d["num_interfaces_ext_mesh"] > 0:
            d["my_neighbors_ext_mesh"] = r.i4()
            d["nibool_interfaces_ext_mesh"] = r.i4()
            d["ibool_interfaces_ext_mesh"] = r.i4()
        r.check(9996)
        # :1050-1146
        if elastic and anisotropy:
            for k in ("c11", "c12", "c13", "c14", "c15", "c16", "c22", "c23", "c24", "c25",
                      "c26", "c33", "c34", "c35", "c36", "c44", "c45", "c46", "c55", "c56",
                      "c66"):
                d[k + "store"] = sized(k + "store", r.f4(), ne, "check the ANISOTROPY switch")
        # no check word follows: the sizes catch a wrong ANISOTROPY switch
        d["ispec_is_inner"] = sized("ispec_is_inner", r.logical(), d["NSPEC_AB"],
                                    "check the ANISOTROPY switch")
        for kind, present in (("acoustic", acoustic), ("elastic", elastic),
                              ("poroelastic", poro)):
            if present:
                inner_outer = sized(f"nspec_inner/outer_{kind}", r.i4(), 2)
                d[f"nspec_inner_{kind}"], d[f"nspec_outer_{kind}"] = (int(inner_outer[0]),
                                                                      int(inner_outer[1]))
                n = d[f"num_phase_ispec_{kind}"] = r.int()
                if n > 0:
                    d[f"phase_ispec_inner_{kind}"] = r.i4()
    finally:
        r.close()
    return d


def to_database(d) -> Database:
    """The solver's database from the records of an elastic slice (acoustic
    and poroelastic elements, PML and anisotropy are outside the path)."""
    nspec, nglob = d["NSPEC_AB"], d["NGLOB_AB"]
    if not d["ispec_is_elastic"].all():
        raise ValueError("only all-elastic slices run on the solver")
    if d.get("NSPEC_CPML", 0) > 0 or "c11store" in d:
        raise ValueError("C-PML and anisotropic slices are outside the solver's path")
    shape = (nspec, 5, 5, 5)
    el = lambda a: np.asarray(a, np.float32).reshape(shape)  # noqa: E731
    kappa, mu, rho = el(d["kappastore"]), el(d["mustore"]), el(d["rhostore"])
    nirr = d["NSPEC_IRREGULAR"]
    irr = np.asarray(d["irregular_element_number"], np.int64)
    irregular = geo = None
    if nirr > 0:
        irregular = np.where(irr > 0, irr - 1, -1).astype(np.int32)
        names = ("xixstore", "xiystore", "xizstore", "etaxstore", "etaystore", "etazstore",
                 "gammaxstore", "gammaystore", "gammazstore", "jacobianstore")
        geo = np.stack([np.asarray(d[k], np.float32).reshape(nirr, 5, 5, 5) for k in names],
                       axis=-1)
    nf = d["num_abs_boundary_faces"]
    if nf > 0:
        abs_ispec = np.asarray(d["abs_boundary_ispec"], np.int32) - 1
        abs_ijk = np.asarray(d["abs_boundary_ijk"], np.int32).reshape(nf, 25, 3) - 1
        abs_jw = np.asarray(d["abs_boundary_jacobian2Dw"], np.float32).reshape(nf, 25)
        abs_normal = np.asarray(d["abs_boundary_normal"], np.float32).reshape(nf, 25, 3)
    else:
        abs_ispec = np.zeros(0, np.int32)
        abs_ijk = np.zeros((0, 25, 3), np.int32)
        abs_jw = np.zeros((0, 25), np.float32)
        abs_normal = np.zeros((0, 25, 3), np.float32)
    vs = np.sqrt(np.maximum(mu / rho, 0.0)).astype(np.float32)
    vp = np.sqrt(np.maximum((kappa + 4.0 / 3.0 * mu) / rho, 0.0)).astype(np.float32)
    return Database(
        box=None, nspec=nspec, nglob=nglob,
        ibool=np.asarray(d["ibool"], np.int32).reshape(shape) - 1,
        xstore=np.asarray(d["xstore"], np.float32), ystore=np.asarray(d["ystore"], np.float32),
        zstore=np.asarray(d["zstore"], np.float32),
        xix_regular=d["xix_regular"], jacobian_regular=d["jacobian_regular"],
        kappa=kappa, mu=mu, rho=rho, rmass=np.asarray(d["rmass"], np.float32),
        rho_vp=el(d["rho_vp"]), rho_vs=el(d["rho_vs"]),
        abs_ispec=abs_ispec, abs_ijk=abs_ijk, abs_jw=abs_jw, abs_normal=abs_normal,
        vp=vp, vs=vs, irregular=irregular, geo=geo)


class _Writer:
    def __init__(self, path):
        self.f = open(path, "wb")

    def rec(self, data: bytes):
        self.f.write(struct.pack("<i", len(data)))
        self.f.write(data)
        self.f.write(struct.pack("<i", len(data)))

    def i4(self, a):
        self.rec(np.ascontiguousarray(a, "<i4").tobytes())

    def f4(self, a):
        self.rec(np.ascontiguousarray(a, "<f4").tobytes())

    def close(self):
        self.f.close()


CPML_ARRAYS = ("d_store_x", "d_store_y", "d_store_z", "k_store_x", "k_store_y", "k_store_z",
               "alpha_store_x", "alpha_store_y", "alpha_store_z")
ANISO_NAMES = ("c11", "c12", "c13", "c14", "c15", "c16", "c22", "c23", "c24", "c25", "c26",
               "c33", "c34", "c35", "c36", "c44", "c45", "c46", "c55", "c56", "c66")
IBELM_NAMES = ("ibelm_xmin", "ibelm_xmax", "ibelm_ymin", "ibelm_ymax", "ibelm_bottom",
               "ibelm_top")


def write_external_mesh(path, db: Database, *, dt=None, free_surface=None, ocean_load=None,
                        cpml=None, interfaces=None, anisotropy=None, ibelm=None):
    """Write an elastic single-slice database in the record order
    read_mesh_databases.f90 reads (Stacey on).  ``rmassx/y/z`` carry the
    Stacey term ``dt/2 C`` when ``dt`` is given, else the plain mass.

    Optional record groups, each read only under the matching switch of
    ``read_external_mesh`` (indices 0-based here, written 1-based):
    - ``free_surface``: (ispec, ijk, jw, normal) of the free-surface faces;
    - ``ocean_load``: ``rmass_ocean_load`` [nglob] (APPROXIMATE_OCEAN_LOAD);
    - ``cpml``: dict with ``NSPEC_CPML``, the three ``CPML_width_*``,
      ``min_distance_between_CPML_parameter``, ``CPML_regions``,
      ``CPML_to_spec``, ``is_CPML`` [nspec], the nine damping arrays and
      ``points_interface_PML_elastic`` (PML_CONDITIONS; the Stacey mass
      records are then absent, as the reader expects);
    - ``interfaces``: (my_neighbors, nibool, ibool_interfaces) of the MPI
      interfaces;
    - ``anisotropy``: dict ``c11`` .. ``c66`` of element arrays (ANISOTROPY);
    - ``ibelm``: dict ``ibelm_xmin`` .. ``ibelm_top`` of element lists."""
    nspec, nglob = db.nspec, db.nglob
    nirr = db.nspec_irregular
    w = _Writer(path)
    try:
        w.i4([nspec])
        w.i4([nglob])
        w.i4([nirr])
        w.i4(np.asarray(db.ibool).reshape(-1) + 1)
        for a in (db.xstore, db.ystore, db.zstore):
            w.f4(a)
        if nirr > 0:
            w.i4(np.where(db.irregular >= 0, db.irregular + 1, 0))
        else:
            w.i4(np.zeros(nspec))
        w.f4([db.xix_regular])
        w.f4([db.jacobian_regular])
        for q in range(10):
            w.f4(db.geo[..., q].reshape(-1) if nirr > 0 else [0.0])
        for a in (db.kappa, db.mu, db.rho):
            w.f4(np.asarray(a).reshape(-1))
        w.i4(np.zeros(nspec))           # ispec_is_acoustic
        w.i4(np.ones(nspec))            # ispec_is_elastic
        w.i4(np.zeros(nspec))           # ispec_is_poroelastic
        w.i4([9999])
        w.f4(db.rmass)
        if ocean_load is not None:
            w.f4(ocean_load)
        w.f4(np.asarray(db.rho_vp).reshape(-1))
        w.f4(np.asarray(db.rho_vs).reshape(-1))
        if cpml is not None:
            w.i4([cpml["NSPEC_CPML"]])
            for k in ("CPML_width_x", "CPML_width_y", "CPML_width_z",
                      "min_distance_between_CPML_parameter"):
                w.f4([cpml[k]])
            if cpml["NSPEC_CPML"] > 0:
                w.i4(cpml["CPML_regions"])
                w.i4(np.asarray(cpml["CPML_to_spec"]) + 1)
                w.i4(np.asarray(cpml["is_CPML"], np.int32))
                for k in CPML_ARRAYS:
                    w.f4(np.asarray(cpml[k]).reshape(-1))
                pts = np.asarray(cpml.get("points_interface_PML_elastic", []), np.int64)
                w.i4([0])                       # nglob_interface_PML_acoustic
                w.i4([pts.size])                # nglob_interface_PML_elastic
                if pts.size:
                    w.i4(pts + 1)
        nf = db.nfaces
        w.i4([nf])
        if nf > 0:
            w.i4(db.abs_ispec + 1)
            w.i4(np.asarray(db.abs_ijk).reshape(-1) + 1)
            w.f4(np.asarray(db.abs_jw).reshape(-1))
            w.f4(np.asarray(db.abs_normal).reshape(-1))
            rm = np.tile(np.asarray(db.rmass, np.float64)[:, None], (1, 3))
            if dt is not None:
                ib = np.asarray(db.ibool).reshape(nspec, -1)
                ijk = np.asarray(db.abs_ijk)
                lp = ijk[..., 0] + 5 * ijk[..., 1] + 25 * ijk[..., 2]
                ig = ib[np.asarray(db.abs_ispec)[:, None], lp]
                e = np.asarray(db.abs_ispec)[:, None]
                rvp = np.asarray(db.rho_vp).reshape(nspec, -1)[e, lp]
                rvs = np.asarray(db.rho_vs).reshape(nspec, -1)[e, lp]
                n = np.asarray(db.abs_normal, np.float64)
                for c in range(3):
                    term = 0.5 * dt * db.abs_jw * (rvp * n[..., c] ** 2 + rvs * (1 - n[..., c] ** 2))
                    np.add.at(rm[:, c], ig.reshape(-1), term.reshape(-1))
            if cpml is None:
                for c in range(3):
                    w.f4(rm[:, c])
        w.i4([9998])
        ib = ibelm or {}
        for k in IBELM_NAMES:           # nspec2D_xmin .. NSPEC2D_TOP
            w.i4([len(ib.get(k, []))])
        for k in IBELM_NAMES:
            if len(ib.get(k, [])):
                w.i4(np.asarray(ib[k]) + 1)
        if free_surface is not None:
            fs_ispec, fs_ijk, fs_jw, fs_n = free_surface
            w.i4([len(fs_ispec)])
            w.i4(np.asarray(fs_ispec) + 1)
            w.i4(np.asarray(fs_ijk).reshape(-1) + 1)
            w.f4(np.asarray(fs_jw).reshape(-1))
            w.f4(np.asarray(fs_n).reshape(-1))
        else:
            w.i4([0])
        w.i4([0])                       # coupling acoustic-elastic
        w.i4([0])                       # coupling acoustic-poroelastic
        w.i4([0])                       # coupling elastic-poroelastic
        w.i4([9997])
        if interfaces is not None:
            nb, nib, ibi = interfaces
            w.i4([len(nb)])
            w.i4([int(np.max(nib))])
            w.i4(nb)
            w.i4(nib)
            w.i4(np.asarray(ibi).reshape(-1) + 1)
        else:
            w.i4([0])                   # num_interfaces_ext_mesh
            w.i4([0])                   # max_nibool_interfaces_ext_mesh
        w.i4([9996])
        if anisotropy is not None:
            for k in ANISO_NAMES:
                w.f4(np.asarray(anisotropy[k]).reshape(-1))
        w.i4(np.ones(nspec))            # ispec_is_inner
        w.i4([nspec, 0])                # nspec_inner_elastic, nspec_outer_elastic
        w.i4([nspec])                   # num_phase_ispec_elastic
        # phase_ispec_inner_elastic(num_phase, 2): column 1 outer (none),
        # column 2 inner elements
        w.i4(np.concatenate([np.zeros(nspec), np.arange(1, nspec + 1)]))
    finally:
        w.close()
