"""The reference's particle output and restart files, written and read in its formats.

  allpartdata#######  (loadd.f90:147-670, loadpart): one direct-access record
      holding np particles, each the sequence of type particle_restart
      (loadd.f90:149-160): six scalars x, y, z, integralv, volume, volume0,
      then 22 arrays of nl reals in PARTICLE_ARRAYS order; FP64 in the
      machine's byte order, no record markers (recl = np (6 + 22 nl) reals).
  Capsule###step#######.txt  (main.f90:461-467): per point of capsule ###
      (1-based) one line '(3E15.7)' of yfp, zfp, xfp -- y first.
  center_velocity.txt  (main.f90:469-471): appended lines '(7E16.8)' of time,
      the centroid of particle 1 and the mean interpolated velocity ulmean,
      vlmean, wlmean of Update_Pos.f90:131-155.
  epsilonxy.txt  (main.f90:474-476): appended lines '(3E16.8)' of time, exy1
      and exy2 of surf_vol.f90:105-125.

Numbers are formatted as a Fortran Ew.d edit descriptor writes them: a
leading "0.", d significant digits, and a signed two-digit exponent after
"E" (a three-digit exponent replaces the "E"), right-justified in w columns.
"""
import os
import re

import numpy as np

PARTICLE_SCALARS = ("x", "y", "z", "integralv", "volume", "volume0")
PARTICLE_ARRAYS = ("xfp", "yfp", "zfp", "dxdt", "dydt", "dzdt", "fxl", "fyl", "fzl", "ul", "vl", "wl",
                   "xfpo", "yfpo", "zfpo", "xfpold", "yfpold", "zfpold", "xfp0", "yfp0", "zfp0", "area")


def allpartdata_name(istep):
    return "allpartdata%07d" % istep


def capsule_txt_name(p, istep):
    """p: 1-based particle number, as in the reference."""
    return "Capsule%03dstep%07d.txt" % (p, istep)


def fortran_e(x, w, d):
    """x as the Fortran edit descriptor Ew.d writes it, e.g. fortran_e(-12.5, 15, 7) == ' -0.1250000E+02'."""
    x = float(x)
    if not np.isfinite(x):
        s = "NaN" if np.isnan(x) else ("-Infinity" if x < 0 else "Infinity")
        return s.rjust(w) if len(s) <= w else "*" * w
    sign = "-" if (x < 0 or (x == 0 and np.signbit(x))) else ""
    a = abs(x)
    if a == 0.0:
        digits, e = "0" * d, 0
    else:
        m, ex = ("%.*e" % (d - 1, a)).split("e")  # d significant digits, correctly rounded
        digits, e = m.replace(".", ""), int(ex) + 1
    exp = ("E%+03d" % e) if abs(e) <= 99 else ("%+04d" % e)
    s = "%s0.%s%s" % (sign, digits, exp)
    return s.rjust(w) if len(s) <= w else "*" * w


def parse_fortran_e(s):
    """Inverse of fortran_e for one field (accepts the exponent without 'E')."""
    t = s.strip()
    m = re.fullmatch(r"([+-]?\d*\.\d*)([+-]\d+)", t)
    if m:
        return float(m.group(1) + "e" + m.group(2))
    return float(t)


def _lines(values, w, d):
    return "".join("".join(fortran_e(v, w, d) for v in row) + "\n" for row in values)


def write_capsule_txt(path, x, y, z):
    """Capsule###step#######.txt: (yfp, zfp, xfp) per point, '(3E15.7)'."""
    rows = np.stack([np.asarray(y, np.float64), np.asarray(z, np.float64), np.asarray(x, np.float64)], axis=1)
    with open(path, "w") as f:
        f.write(_lines(rows, 15, 7))


def read_capsule_txt(path):
    """Returns (x, y, z) from a Capsule###step#######.txt file."""
    vals = []
    with open(path) as f:
        for line in f:
            if line.strip():
                vals.append([parse_fortran_e(line[15 * q:15 * (q + 1)]) for q in range(3)])
    a = np.asarray(vals, np.float64).reshape(-1, 3)
    return a[:, 2].copy(), a[:, 0].copy(), a[:, 1].copy()


def append_center_velocity(path, time, centroid, mean_velocity):
    """center_velocity.txt: time, x, y, z of particle 1, ulmean, vlmean, wlmean ('(7E16.8)')."""
    with open(path, "a") as f:
        f.write(_lines([[time, *centroid, *mean_velocity]], 16, 8))


def append_epsilonxy(path, time, exy1, exy2):
    """epsilonxy.txt: time, exy1, exy2 ('(3E16.8)')."""
    with open(path, "a") as f:
        f.write(_lines([[time, exy1, exy2]], 16, 8))


def write_allpartdata(path, scalars, arrays):
    """scalars: [np, 6] in PARTICLE_SCALARS order; arrays: [np, 22, nl] in PARTICLE_ARRAYS order."""
    scalars = np.asarray(scalars, np.float64)
    arrays = np.asarray(arrays, np.float64)
    npart = scalars.shape[0]
    if scalars.shape != (npart, 6) or arrays.ndim != 3 or arrays.shape[:2] != (npart, 22):
        raise ValueError("scalars must be [np, 6] and arrays [np, 22, nl]")
    rec = np.concatenate([scalars, arrays.reshape(npart, -1)], axis=1)
    with open(path, "wb") as f:
        f.write(np.ascontiguousarray(rec).tobytes())


def read_allpartdata(path, npart, nl):
    """Returns (scalars [np, 6], arrays [np, 22, nl]); the file must hold exactly one record."""
    skip = 6 + 22 * nl
    rec = np.fromfile(path, dtype=np.float64)
    if rec.size != npart * skip:
        raise ValueError("%s holds %d reals, expected np (6 + 22 nl) = %d" % (path, rec.size, npart * skip))
    rec = rec.reshape(npart, skip)
    return rec[:, :6].copy(), rec[:, 6:].reshape(npart, 22, nl).copy()


def particle_state(offsets, positions, velocity=None, force=None, area=None, volume=None, volume0=None,
                   initial=None):
    """Per-capsule record of allpartdata from the library's concatenated arrays.

    positions, velocity, force: (x, y, z) triples of concatenated point arrays
    (capsule after capsule); initial: the positions at the start (xfp0..).
    The centroid goes to x, y, z; dxdt.. and ul.. both take the interpolated
    velocity (forward Euler makes them equal); xfpo.. and xfpold.. take the
    current positions, and integralv is zero: this path keeps no older states.
    Capsules must have equal point counts (nl), as the reference's do.
    """
    off = np.asarray(offsets, np.int64)
    npart = off.size - 1
    nl = int(off[1] - off[0]) if npart else 0
    if npart and np.any(np.diff(off) != nl):
        raise ValueError("allpartdata needs equal point counts per capsule")
    zero = [np.zeros(off[-1]) for _ in range(3)]
    vel = velocity if velocity is not None else zero
    frc = force if force is not None else zero
    ini = initial if initial is not None else positions
    ar = area if area is not None else np.zeros(off[-1])
    cols = [*positions, *vel, *frc, *vel, *positions, *positions, *ini, ar]
    arrays = np.stack([np.asarray(c, np.float64).reshape(npart, nl) for c in cols], axis=1)
    scalars = np.zeros((npart, 6))
    scalars[:, 0:3] = np.stack([np.asarray(p, np.float64).reshape(npart, nl).mean(axis=1) for p in positions], 1)
    if volume is not None:
        scalars[:, 4] = volume
    scalars[:, 5] = volume0 if volume0 is not None else scalars[:, 4]
    return scalars, arrays


def write_step_outputs(directory, istep, time, offsets, positions, velocity, exy1, exy2):
    """The every-100-steps outputs of main.f90:455-476 for capsules 1..np:
    Capsule###step#######.txt per capsule, and per capsule one line each in
    center_velocity.txt (particle 1's centroid; the mean velocity, ulmean..,
    and exy1, exy2 of the last capsule, the values the reference's globals
    hold after its loops) and epsilonxy.txt."""
    off = np.asarray(offsets, np.int64)
    npart = off.size - 1
    os.makedirs(directory, exist_ok=True)
    cen1 = [float(np.sum(p[off[0]:off[1]]) / (off[1] - off[0])) for p in positions]
    last = slice(off[npart - 1], off[npart])
    umean = [float(np.sum(u[last]) / (off[npart] - off[npart - 1])) for u in velocity]
    for p in range(npart):
        s = slice(off[p], off[p + 1])
        write_capsule_txt(os.path.join(directory, capsule_txt_name(p + 1, istep)),
                          positions[0][s], positions[1][s], positions[2][s])
        append_center_velocity(os.path.join(directory, "center_velocity.txt"), time, cen1, umean)
        append_epsilonxy(os.path.join(directory, "epsilonxy.txt"), time, exy1, exy2)
