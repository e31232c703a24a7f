"""Restart files of the reference, written and read from the device state.

Formats (Fortran formatted, list-directed after '#' comment lines, which `titols` skips):

* density file -- He_statics/printout.f90:52-69, read by He_statics/readen.f90:71-84 (mode 0) and
  by Dynamics_TDDFT/readenc.f90:66-88 (mode 0, density branch):
      '#' comment lines
      xmax ymax zmax hx hy hz nx ny nz limp ximp yimp zimp
      den(nx,ny,nz)                      (column-major, x fastest)
* wave-function file -- Dynamics_TDDFT/printoutc.f90:24-79, read by readenc.f90:90-110 (mode 2):
      '#' header with iteration, time step, potentials, energies, observables
      xmax ymax zmax hx hy hz nx ny nz
      N_imp
      rimp(N_imp,3)
      vimp(N_imp,3)
      psi(nx,ny,nz)                      (complex, '(re,im)')

The reader accepts what Fortran list-directed output produces: values separated by blanks,
commas or line ends, repeat counts 'r*value', complex constants '(re, im)', 'D' exponents and
logical T/F.  Values are written with 17 significant digits, so a file written here and read back
(by this reader or by the reference's list-directed reads) reproduces binary64 exactly.
"""
import re

import numpy as np

_TOKEN = re.compile(r"(?:\d+\*)?\(\s*[^(),\s]+\s*,\s*[^(),\s]+\s*\)|[^\s,]+")


def _num(t):
    return float(t.replace("D", "E").replace("d", "e"))


def _values(text):
    """Expand the list-directed values of `text` (comment lines already removed)."""
    out = []
    for tok in _TOKEN.findall(text):
        rep = 1
        m = re.match(r"^(\d+)\*(.+)$", tok)
        if m:
            rep, tok = int(m.group(1)), m.group(2)
        if tok.startswith("("):
            re_, im_ = tok[1:-1].split(",")
            v = complex(_num(re_.strip()), _num(im_.strip()))
        elif tok.upper() in ("T", ".TRUE.", "F", ".FALSE."):
            v = tok.upper() in ("T", ".TRUE.")
        else:
            v = _num(tok)
        out.extend([v] * rep)
    return out


def _body(path):
    """The file after its leading '#' lines (titols.f90: skip lines whose first column is '#')."""
    lines = open(path).read().splitlines()
    k = 0
    while k < len(lines) and lines[k][:1] == "#":
        k += 1
    return "\n".join(lines[k:])


def _fmt(v):
    if isinstance(v, (bool, np.bool_)):
        return "T" if v else "F"
    if isinstance(v, (int, np.integer)):
        return str(int(v))
    if isinstance(v, complex) or np.iscomplexobj(v):
        return f"({v.real:.16E},{v.imag:.16E})"
    return f"{float(v):.16E}"


def _write_list(f, values, per_line=3):
    vals = list(values)
    for i in range(0, len(vals), per_line):
        f.write(" " + " ".join(_fmt(v) for v in vals[i:i + per_line]) + "\n")


def write_density(path, w, den, iteration=0, limp=False, rimp=(0.0, 0.0, 0.0), comment=""):
    """He_statics printout (density) for workload w."""
    hx, hy, hz = w.h
    with open(path, "w") as f:
        f.write(f"#  Density after {iteration} iterations {comment}\n#  \n")
        _write_list(f, [w.xmax, w.ymax, w.zmax, hx, hy, hz, w.nx, w.ny, w.nz, bool(limp),
                        *[float(c) for c in rimp]], per_line=13)
        _write_list(f, np.asarray(den, dtype=np.float64).ravel(order="F"))


def read_density(path):
    """(header dict, den (nx,ny,nz) Fortran order)."""
    v = _values(_body(path))
    xmax, ymax, zmax, hx, hy, hz = v[:6]
    nx, ny, nz = (int(round(x)) for x in v[6:9])
    limp = bool(v[9])
    rimp = tuple(float(x) for x in v[10:13])
    n = nx * ny * nz
    den = np.asarray(v[13:13 + n], dtype=np.float64)
    if den.size != n:
        raise ValueError(f"{path}: {den.size} density values for a {nx}x{ny}x{nz} grid")
    hdr = dict(xmax=xmax, ymax=ymax, zmax=zmax, hx=hx, hy=hy, hz=hz, nx=nx, ny=ny, nz=nz,
               limp=limp, rimp=rimp)
    return hdr, den.reshape((nx, ny, nz), order="F")


def write_wavefunction(path, w, psi, rimp, vimp, iteration=0, time_ps=0.0, energies=None,
                       observables=None):
    """Dynamics_TDDFT printoutc for workload w: psi (nx,ny,nz) complex, rimp/vimp (N_imp,3)."""
    hx, hy, hz = w.h
    rimp = np.asarray(rimp, dtype=np.float64).reshape(-1, 3)
    vimp = np.asarray(vimp, dtype=np.float64).reshape(-1, 3)
    e = energies or {}
    o = observables or {}
    with open(path, "w") as f:
        f.write("#  \n")
        f.write(f"#  Density after {iteration:15d} iterations\n")
        f.write(f"#  Actual deltatps....:{w.deltatps:20.10E}\n")
        f.write(f"#  Total evolution time(ps)...:{time_ps:20.12E}\n")
        for k in range(rimp.shape[0]):
            f.write("#  Impurity-helium potential.........:  Morse\n")
            f.write(f"#  r_cutoff_gs:{w.pot_rcut:16.8E}\n#  umax_gs....:{w.pot_umax:16.8E}\n")
        f.write("#  xcm,ycm,zcm:" + "".join(f"{o.get(k, 0.0):16.8E}" for k in ("xcm", "ycm", "zcm")) + "\n")
        f.write(f"#  NParticles.:{o.get('n', 0.0):16.8E}\n")
        for label, key in (("Ekin.......", "ekin4"), ("Elj........", "elj4"),
                           ("Ealphas....", "ealphas"), ("Ecorr......", "ecor4"),
                           ("Esolid.....", "esolid"), ("Ekinx......", "ekinx"),
                           ("Eimpu......", "eimpu"), ("Etot.......", "etot")):
            f.write(f"#  {label}:{e.get(key, 0.0):16.8E}\n")
        f.write("#  <Lx,y,z>...:" + "".join(f"{o.get(k, 0.0):16.8E}" for k in ("lx", "ly", "lz")) + "\n")
        f.write("#  <x2,y2,z2>.:" + "".join(f"{o.get(k, 0.0):16.8E}" for k in ("r2x", "r2y", "r2z")) + "\n")
        f.write("#  <Vcom_x,y,z>...:" + "".join(f"{o.get(k, 0.0):16.8E}" for k in ("vcomx", "vcomy", "vcomz")) + "\n")
        f.write("#  \n")
        _write_list(f, [w.xmax, w.ymax, w.zmax, hx, hy, hz, w.nx, w.ny, w.nz], per_line=9)
        _write_list(f, [rimp.shape[0]])
        _write_list(f, rimp.ravel(order="F"))
        _write_list(f, vimp.ravel(order="F"))
        _write_list(f, np.asarray(psi, dtype=np.complex128).ravel(order="F"), per_line=2)


def read_wavefunction(path, n_imp):
    """readenc mode 2: (header dict, rimp (N_imp,3), vimp (N_imp,3), psi (nx,ny,nz)).  A file
    with a different impurity count is rejected, as readenc.f90:98-102 stops on it."""
    v = _values(_body(path))
    xmax, ymax, zmax, hx, hy, hz = (float(x.real if isinstance(x, complex) else x) for x in v[:6])
    nx, ny, nz = (int(round(x)) for x in v[6:9])
    k = 9
    n0 = int(round(v[k]))
    k += 1
    if n0 != n_imp:
        raise ValueError(f"Number of impurities are inconsistent: {n_imp} {n0}")
    rimp = np.asarray(v[k:k + 3 * n0], dtype=np.float64).reshape((n0, 3), order="F")
    k += 3 * n0
    vimp = np.asarray(v[k:k + 3 * n0], dtype=np.float64).reshape((n0, 3), order="F")
    k += 3 * n0
    n = nx * ny * nz
    psi = np.asarray(v[k:k + n], dtype=np.complex128)
    if psi.size != n:
        raise ValueError(f"{path}: {psi.size} psi values for a {nx}x{ny}x{nz} grid")
    hdr = dict(xmax=xmax, ymax=ymax, zmax=zmax, hx=hx, hy=hy, hz=hz, nx=nx, ny=ny, nz=nz)
    return hdr, rimp, vimp, psi.reshape((nx, ny, nz), order="F")


def snapshot(ctx, path, npart, iteration=0, time_ps=0.0):
    """printoutc of a device context: downloads psi, rimp, vimp, computes energy() and the
    droplet observables on the device, and writes the wave-function file."""
    w = ctx.w
    psi = ctx.download("psi")
    rimp = ctx.download("rimp") if w.n_imp else np.zeros((0, 3))
    vimp = ctx.download("vimp") if w.n_imp else np.zeros((0, 3))
    e = ctx.energy()
    o = ctx.observables(npart)
    write_wavefunction(path, w, psi, rimp, vimp, iteration, time_ps, e, o)


def restore(ctx, path):
    """readenc mode 2 into a device context: psi, den = conjg(psi)*psi, rimp, vimp."""
    w = ctx.w
    hdr, rimp, vimp, psi = read_wavefunction(path, w.n_imp)
    if (hdr["nx"], hdr["ny"], hdr["nz"]) != (w.nx, w.ny, w.nz):
        raise ValueError("restart grid differs from the context's grid")
    ctx.upload("psi", psi)
    ctx.upload("den", (np.conj(psi) * psi).real)
    if w.n_imp:
        ctx.upload("rimp", rimp)
        ctx.upload("vimp", vimp)
    return hdr
