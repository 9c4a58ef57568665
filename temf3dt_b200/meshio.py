"""Reference file formats: MEDIT ``.mesh``, keyword ``.cntl``, ``.field``.

Host-side readers/writers with the reference's conventions
(model_mesh, src/FETD_FWD.f90:112-166; model_ctl, :284-497; solution_output's
``.field`` row, :1623).  They produce plain arrays for the C ABI.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

MU0 = 3.141592653589793238462643383279502884197 * 4.0e-7   # src/FETD_FWD.f90:15
EPS0 = 8.8541878176e-12                                     # src/FETD_FWD.f90:16


def _num(tok: str) -> float:
    return float(tok.replace("d", "e").replace("D", "E"))


@dataclass
class Mesh:
    nod_cor: np.ndarray            # (N,3) float64
    tet_vex: np.ndarray            # (T,4) 1-based
    tet_phy: np.ndarray            # (T,)
    src_vex: np.ndarray            # (S,2) 1-based (Edges with non-zero tag)
    src_phy: np.ndarray            # (S,)


def read_mesh(path: str) -> Mesh:
    """MEDIT ``.mesh``: sections keyed by the first five letters of their name."""
    with open(path, "r") as fh:
        lines = fh.read().splitlines()
    nod = tet = phy = None
    sv = np.zeros((0, 2), dtype=np.int64)
    sp = np.zeros(0, dtype=np.int64)
    i = 0
    while i < len(lines):
        t = lines[i].split()
        w = t[0][:5] if t else ""
        if w in ("Verti", "Edges", "Trian", "Tetra"):
            cnt = int(lines[i + 1].split()[0])
            body = lines[i + 2:i + 2 + cnt]
            i += 2 + cnt
            if w == "Verti":
                a = np.array([_num(x) for ln in body for x in ln.split()[:3]], dtype=np.float64)
                nod = a.reshape(cnt, 3)
            elif w == "Edges":
                a = np.array(" ".join(body).split(), dtype=np.int64).reshape(cnt, 3)
                keep = a[:, 2] != 0
                sv, sp = a[keep, :2], a[keep, 2]
            elif w == "Tetra":
                a = np.array(" ".join(body).split(), dtype=np.int64).reshape(cnt, 5)
                tet, phy = a[:, :4], a[:, 4]
            continue
        i += 1
    if nod is None or tet is None:
        raise ValueError("%s: no Vertices/Tetrahedra section" % path)
    return Mesh(nod, tet, phy, sv, sp)


def write_mesh(path: str, mesh: Mesh) -> None:
    """Write a MEDIT ``.mesh`` that ``read_mesh`` (and the reference) accept."""
    with open(path, "w") as fh:
        fh.write(" MeshVersionFormatted 2\n Dimension\n 3\n Vertices\n %d\n" % len(mesh.nod_cor))
        for k, (x, y, z) in enumerate(mesh.nod_cor):
            fh.write(" %.17g %.17g %.17g 0\n" % (x, y, z))
        if len(mesh.src_vex):
            fh.write(" Edges\n %d\n" % len(mesh.src_vex))
            for (a, b), p in zip(mesh.src_vex, mesh.src_phy):
                fh.write(" %d %d %d\n" % (a, b, p))
        fh.write(" Tetrahedra\n %d\n" % len(mesh.tet_vex))
        for (a, b, c, d), p in zip(mesh.tet_vex, mesh.tet_phy):
            fh.write(" %d %d %d %d %d\n" % (a, b, c, d, p))
        fh.write(" End\n")


@dataclass
class Control:
    rec_cor: np.ndarray = None
    rec_charac: float = 10.0
    domains: List[tuple] = field(default_factory=list)   # (phys, sigma, eps_r, mu_r)
    bound_cond: int = 0
    src_num: int = 0
    source_type: int = 1
    pulse_type: int = 1
    t0: float = 0.0
    current: float = 1.0
    sp_mthd: int = 0
    sp_division: int = 0
    time_maximum: float = 0.0
    sp_double: int = 0
    sp_dblesize: int = 2
    output: np.ndarray = field(default_factory=lambda: np.zeros(9, dtype=bool))
    time_points: Optional[np.ndarray] = None
    vtkout: int = 0
    vtk_times: Optional[np.ndarray] = None
    # anisotropic media (src/FETD_FWD.f90:368-410): per domain
    # (phys, (s1, s2, s3), (a1, a2, a3) degrees) for sigma, eps_r and mu_r
    aniso_domains: List[tuple] = field(default_factory=list)


def _parse(line: str):
    s = line.replace("\t", " ")
    st = s.strip()
    if not st or st[0] in "%!":
        return None
    if ":" not in s:
        return ("", "")
    k = s.index(":")
    v = s[k + 1:]
    for ch in "%!":
        j = v.find(ch)
        if j > 0:
            v = v[:j]
    return s[:k].strip().lower(), v.strip()


def read_cntl(path: str) -> Control:
    """Keyword file of model_ctl (isotropic media; src/FETD_FWD.f90:311-497)."""
    c = Control()
    with open(path) as fh:
        L = fh.read().splitlines()
    i = 0
    while i < len(L):
        pc = _parse(L[i]); i += 1
        if pc is None:
            continue
        k, v = pc
        if k == "receivers":
            n = int(v.split()[0]); c.rec_cor = np.array([[_num(t) for t in L[i + q].split()[:3]] for q in range(n)]); i += n
        elif k == "rec_charac":
            c.rec_charac = _num(v.split()[0])
        elif k == "isotropic":
            n = int(v.split()[0])
            for q in range(n):
                t = L[i + q].split()
                c.domains.append((int(t[0]), _num(t[1]), _num(t[2]), _num(t[3])))
            i += n
        elif k == "anisotropic":
            n = int(v.split()[0])
            rows = [[_num(t) for t in L[i + q].split()[:7]] for q in range(3 * n)]
            i += 3 * n
            for q in range(n):
                s, e, m = rows[3 * q], rows[3 * q + 1], rows[3 * q + 2]
                c.aniso_domains.append((int(s[0]), (tuple(s[1:4]), tuple(s[4:7])), (tuple(e[1:4]), tuple(e[4:7])),
                                        (tuple(m[1:4]), tuple(m[4:7]))))
        elif k == "boundary condition":
            c.bound_cond = int(v.split()[0])
        elif k == "source":
            c.src_num = int(v.split()[0])
            t = L[i].split(); i += 1
            c.source_type, c.pulse_type, c.t0, c.current = int(t[0]), int(t[1]), _num(t[2]), _num(t[3])
        elif k == "sp_mthd":
            c.sp_mthd = int(v.split()[0])
        elif k == "sp_division":
            c.sp_division = int(v.split()[0])
        elif k == "time_maximum":
            c.time_maximum = _num(v.split()[0])
        elif k == "sp_double":
            c.sp_double = int(v.split()[0])
        elif k == "sp_dblesize":
            c.sp_dblesize = int(v.split()[0])
        elif k == "output":
            c.output = np.array([int(x) == 1 for x in L[i].split()[:9]]); i += 1
        elif k == "time_points":
            n = int(v.split()[0]); c.time_points = np.array([_num(L[i + q].split()[0]) for q in range(n)]); i += n
        elif k == "vtkout":
            c.vtkout = int(v.split()[0])
            if c.vtkout > 0:
                c.vtk_times = np.array([_num(L[i + q].split()[0]) for q in range(c.vtkout)])
            i += max(c.vtkout, 0)
    if c.rec_cor is None or not len(c.rec_cor) or not (c.domains or c.aniso_domains) or not c.src_num \
            or not c.sp_mthd \
            or not c.sp_division or abs(c.time_maximum) < 1e-20 or not c.sp_double or not c.output.any():
        raise ValueError("%s: incomplete control file (src/FETD_FWD.f90:490-497)" % path)
    return c


def write_cntl(path: str, c: Control) -> None:
    with open(path, "w") as fh:
        fh.write("receivers: %d\n" % len(c.rec_cor))
        for p in c.rec_cor:
            fh.write("%.10g %.10g %.10g\n" % tuple(p))
        fh.write("\nrec_charac: %.10g\n" % c.rec_charac)
        if c.aniso_domains:
            fh.write("\nanisotropic: %d\n" % len(c.aniso_domains))
            for phys, *parts in c.aniso_domains:
                for vals, ang in parts:  # sigma, eps_r, mu_r lines
                    fh.write("%d %s %s\n" % (phys, " ".join("%.10g" % v for v in vals),
                                              " ".join("%.10g" % a for a in ang)))
        else:
            fh.write("\nisotropic: %d\n" % len(c.domains))
            for d in c.domains:
                fh.write("%d %.10g %.10g %.10g\n" % d)
        fh.write("\nboundary condition: %d\n" % c.bound_cond)
        fh.write("\n! TYPE 1 - STEPON / TYPE 2 - IMPULSE / TYPE 3 - STEPOFF\nsource: 1\n")
        fh.write("%d %d %.10g %.10g\n" % (c.source_type, c.pulse_type, c.t0, c.current))
        fh.write("\nsp_mthd: 2\nsp_division: %d\ntime_maximum: %.10g\n" % (c.sp_division, c.time_maximum))
        fh.write("sp_double: %d\nsp_dblesize: %d\n" % (c.sp_double, c.sp_dblesize))
        fh.write("\n! ex ey ez dx dy dz bx by bz\noutput:\n%s\n" % " ".join(str(int(b)) for b in c.output))
        if c.time_points is not None:
            fh.write("\ntime_points: %d\n" % len(c.time_points))
            for t in c.time_points:
                fh.write("%.10g\n" % t)
        if c.vtk_times is not None and len(c.vtk_times):
            fh.write("\nvtkout: %d\n" % len(c.vtk_times))
            for t in c.vtk_times:
                fh.write("%.10g\n" % t)
        else:
            fh.write("\nvtkout: 0\n")


def rotation(ang_deg) -> np.ndarray:
    """dm = dx dy dz of the anisotropic media (src/FETD_FWD.f90:387-390),
    angles in degrees.  The reference's z factor carries cos of the second
    angle at its (2,2) entry, and so does this one (same tensors as the
    reference)."""
    a1, a2, a3 = np.radians(np.asarray(ang_deg, dtype=np.float64))
    dx = np.array([[1.0, 0.0, 0.0], [0.0, np.cos(a1), -np.sin(a1)], [0.0, np.sin(a1), np.cos(a1)]])
    dy = np.array([[np.cos(a2), 0.0, np.sin(a2)], [0.0, 1.0, 0.0], [-np.sin(a2), 0.0, np.cos(a2)]])
    dz = np.array([[np.cos(a3), -np.sin(a3), 0.0], [np.sin(a3), np.cos(a2), 0.0], [0.0, 0.0, 1.0]])
    return dx @ dy @ dz


def media_tensors_per_tet(tet_phy: np.ndarray, ctl: Control):
    """sig_a3d and mag_a3d per tet as (n_tets, 9) row-major arrays
    (src/FETD_FWD.f90:381-409; mag includes mu0)."""
    sig = np.full((len(tet_phy), 9), np.nan)
    mu = np.full((len(tet_phy), 9), np.nan)
    for phys, (sv, sa), _eps, (mv, ma) in ctl.aniso_domains:
        m = tet_phy == phys
        dm = rotation(sa)
        sig[m] = (dm @ np.diag(sv) @ dm.T).reshape(9)
        dm = rotation(ma)
        mu[m] = (dm @ np.diag(mv) @ dm.T).reshape(9) * MU0
    if np.isnan(sig).any():
        raise ValueError("error - physical domain not found!")
    return sig, mu


def media_per_tet(tet_phy: np.ndarray, ctl: Control):
    """sig_3d / mag_3d per tet (src/FETD_FWD.f90:347-364)."""
    sig = np.full(len(tet_phy), np.nan)
    mu = np.full(len(tet_phy), np.nan)
    for phys, s, _eps, mur in ctl.domains:
        m = tet_phy == phys
        sig[m] = s
        mu[m] = mur * MU0
    if np.isnan(sig).any():
        raise ValueError("error - physical domain not found!")
    return sig, mu


def fortran_e(v: float, w: int = 15, d: int = 5) -> str:
    """Fortran Ew.d: [-]0.ddddd E+ee right-justified in w columns (a
    three-digit exponent drops the E)."""
    v = float(v)
    if v != v:
        s = "NaN"
    elif v in (float("inf"), float("-inf")):
        s = "Infinity" if v > 0 else "-Infinity"
    elif v == 0.0:
        s = "0." + "0" * d + "E+00"
    else:
        t = "%.*E" % (d - 1, abs(v))
        mant, ex = t.split("E")
        e = int(ex) + 1
        digits = mant.replace(".", "")
        es = ("E%+03d" % e) if abs(e) < 100 else ("%+04d" % e)
        s = ("-" if v < 0 else "") + "0." + digits + es
    return s.rjust(w)


def write_field(path: str, steps, times, fields: np.ndarray, output_mask: np.ndarray) -> None:
    """``.field`` rows: step, time, then the selected components per receiver
    (src/FETD_FWD.f90:1623, format i6, e15.5, 2x, rec*(n e15.5, 2x)), numbers
    as Fortran's E15.5 writes them."""
    sel = np.nonzero(output_mask)[0]
    with open(path, "w") as fh:
        for i, (s, t) in enumerate(zip(steps, times)):
            parts = ["%6d%s  " % (s, fortran_e(t))]
            for r in range(fields.shape[1]):
                parts.append("".join(fortran_e(v) for v in fields[i, r, sel]) + "  ")
            fh.write("".join(parts).rstrip() + "\n")


def read_field(path: str) -> np.ndarray:
    rows = []
    with open(path) as fh:
        for ln in fh:
            t = ln.split()
            if t:
                rows.append([float(v) for v in t])
    return np.array(rows)
