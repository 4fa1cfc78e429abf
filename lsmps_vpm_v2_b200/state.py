"""2D particle-state CSV files in the reference's format.

`read_particle_state` follows initialization::read_2d_particle
(src/initialization/initialization.cpp:561-680): the header line is skipped,
every row is split at commas and each field converted with std::stod
semantics (the longest leading decimal number, so an "a|b|c" neighbour list
reads as a), and the columns are taken by position

    xp, yp, gpz, vor, up, vp, sp, active, chi[, pressure, ngh_num, ngh_ID]
    0   1   2    3    4   5   6   7       8      9         10       11

`active` is true when its value is non-zero. The particle level is computed
only when sigma and max_level are given, as the reference does from
Pars::sigma and Pars::max_level (initialization.cpp:661-667).

`write_particle_state` follows save_data::save_par_state_2D with type 0
(src/save_data/state_data.cpp:336-385): the same header and column order,
velocities written relative to the body velocity, numbers in the stream's
general format with `precision` significant digits (12 in the reference's
writer; files written by older builds used the stream default of 6), and the
optional pressure / neighbour-count / neighbour-list columns.
"""
from __future__ import annotations

import re

import numpy as np

HEADER = ("xp", "yp", "gpz", "vor", "up", "vp", "sp", "active", "chi")
_NUM = re.compile(r"\s*[+-]?(?:(?:\d+\.?\d*|\.\d+)(?:[eE][+-]?\d+)?|inf(?:inity)?|nan)", re.IGNORECASE)


def _stod(entry: str) -> float:
    """std::stod: the longest leading number (leading whitespace skipped);
    raises ValueError where stod throws std::invalid_argument."""
    m = _NUM.match(entry)
    if not m:
        raise ValueError(f"not a number: {entry!r}")
    return float(m.group(0))


def read_particle_state(path: str, sigma: float | None = None, max_level: int | None = None) -> dict:
    """Particles of a 2D state file as arrays: x, y, gz, vorticity, u, v, s,
    active (uint8), chi, pressure (when the file has that column) and level
    (when sigma and max_level are given)."""
    cols: dict[int, list[float]] = {k: [] for k in range(10)}
    with open(path, "r", newline="") as f:
        f.readline()   # header
        for line in f:
            line = line.rstrip("\r\n")
            if not line:
                continue
            fields = line.split(",")
            for k, entry in enumerate(fields[:10]):
                cols[k].append(_stod(entry))
    n = len(cols[0])
    for k in range(8):
        if len(cols[k]) != n:
            raise ValueError(f"{path}: column {k} has {len(cols[k])} of {n} values")
    out = {
        "x": np.asarray(cols[0], dtype=np.float64),
        "y": np.asarray(cols[1], dtype=np.float64),
        "gz": np.asarray(cols[2], dtype=np.float64),
        "vorticity": np.asarray(cols[3], dtype=np.float64),
        "u": np.asarray(cols[4], dtype=np.float64),
        "v": np.asarray(cols[5], dtype=np.float64),
        "s": np.asarray(cols[6], dtype=np.float64),
        "active": (np.asarray(cols[7], dtype=np.float64) != 0.0).astype(np.uint8),
    }
    if len(cols[8]) == n:
        out["chi"] = np.asarray(cols[8], dtype=np.float64)
    if len(cols[9]) == n and n > 0:
        out["pressure"] = np.asarray(cols[9], dtype=np.float64)
    if sigma is not None and max_level is not None:
        lvl = np.empty(n, dtype=np.int32)
        for i, sp in enumerate(out["s"]):
            level, mul = int(max_level), int((sp + sigma / 100.0) / sigma)   # C++ int conversion truncates
            while mul != 1 and mul != 0:
                level -= 1
                mul //= 2
            lvl[i] = level
        out["level"] = lvl
    return out


def _g(v: float, precision: int) -> str:
    """One number as an ostream with precision(p) and the default float
    format writes it (printf %.{p}g)."""
    return format(float(v), f".{precision}g")


def write_particle_state(path: str, p: dict, precision: int = 12, ubody: float = 0.0, vbody: float = 0.0,
                         pressure: np.ndarray | None = None, ngh_num: np.ndarray | None = None,
                         ngh_ids: list | None = None) -> None:
    """Write particles p (keys as read_particle_state returns; chi defaults to
    zero) in the reference's 2D state format."""
    n = int(np.asarray(p["x"]).size)
    chi = p.get("chi")
    if chi is None:
        chi = np.zeros(n)
    header = ",".join(HEADER)
    if pressure is not None:
        header += ",pressure"
    if ngh_num is not None:
        header += ",ngh_num"
    if ngh_ids is not None:
        header += ",ngh_ID"
    rows = [header]
    x, y, gz, w = p["x"], p["y"], p["gz"], p["vorticity"]
    u, v, s, act = p["u"], p["v"], p["s"], p["active"]
    for i in range(n):
        fields = [_g(x[i], precision), _g(y[i], precision), _g(gz[i], precision), _g(w[i], precision),
                  _g(u[i] - ubody, precision), _g(v[i] - vbody, precision), _g(s[i], precision),
                  "1" if act[i] else "0", _g(chi[i], precision)]
        if pressure is not None:
            fields.append(_g(pressure[i], precision))
        if ngh_num is not None:
            fields.append(str(int(ngh_num[i])))
        if ngh_ids is not None:
            fields.append("|".join(str(int(j)) for j in ngh_ids[i]))
        rows.append(",".join(fields))
    with open(path, "w", newline="") as f:
        f.write("\n".join(rows) + "\n")
