"""Restart files: the reference's text configuration and an exact binary side-car.

``write_conf`` writes the ``conf_new`` file of store_config.f90:20-67 (mode 2,
no STARS, no explicit wall atoms) field by field in the reference's fixed
formats, and ``read_conf`` reads a ``conf_old`` the way init_config.f90:104-209
does, so that a run can start from the reference's restart file and the
reference can start from one written here.  The text format keeps 7 decimals
(positions ``i3,3f13.7``; velocities and accelerations ``3f15.7``), so a
restart through it is not exact; ``write_state``/``read_state`` keep every
FP64 bit of the state for an exact resume (layout below).

Binary side-car (little endian):
    8 bytes   magic ``b"MFASTATE"``
    int32     version (2; version 1 files, without the next two fields, are read too)
    int32     n (particles)
    int64     i_time (the step counter)
    int32     bin_type (the list rule: 0 binning, 1 my_binning)
    int32     reserved (0)
    then      r0, v, a as n x 3 float64 (particle-major, xyz contiguous),
              mic as n x 3 int32 (periodic image counters), a_type as n int32.
"""
from __future__ import annotations

import struct

import numpy as np

MAGIC = b"MFASTATE"
VERSION = 2
N_ORDER = 2          # mfa_common.f90:70 (predictor order kept for the top wall)


def _f(x: float, w: int, d: int) -> str:
    """Fortran Fw.d: right-justified, d decimals, asterisks when it does not fit."""
    s = f"{x:{w}.{d}f}"
    return "*" * w if len(s) > w else s


def _i(k: int, w: int) -> str:
    """Fortran Iw."""
    s = f"{int(k):{w}d}"
    return "*" * w if len(s) > w else s


def write_conf(path: str, r0, v, a, a_type, n_mon: int, n_chain: int, n_mon_d: int = 0,
               n_chain_d: int = 0, n_cell_w=(0, 0), walls: dict | None = None, dt: float = 0.005) -> None:
    """conf_new as store_config.f90:20-67 writes it.

    walls: the moving-wall block that follows the accelerations
    (store_config.f90:55-66): ``r0_twall`` (3), ``rx_twall`` (3 x n_order, the
    derivatives times dt^order as the reference keeps them; written divided by
    dt^order), ``pbc_twall`` (3 int), ``r0_bwall`` (3), ``pbc_bwall`` (3 int),
    ``r0_spring_twall`` (3), ``s_force_grad`` (3 int).  Zeros when omitted
    (no moving top wall)."""
    r0 = np.asarray(r0, dtype=np.float64).reshape(-1, 3)
    v = np.asarray(v, dtype=np.float64).reshape(-1, 3)
    a = np.asarray(a, dtype=np.float64).reshape(-1, 3)
    a_type = np.asarray(a_type).reshape(-1)
    n = r0.shape[0]
    if v.shape[0] != n or a.shape[0] != n or a_type.shape[0] != n:
        raise ValueError("r0, v, a and a_type must describe the same particles")
    w = {"r0_twall": np.zeros(3), "rx_twall": np.zeros((3, N_ORDER)), "pbc_twall": np.zeros(3, int),
         "r0_bwall": np.zeros(3), "pbc_bwall": np.zeros(3, int), "r0_spring_twall": np.zeros(3),
         "s_force_grad": np.zeros(3, int)}
    if walls:
        w.update({k: np.asarray(x) for k, x in walls.items()})
    vec = lambda x: "".join(_f(float(c), 15, 7) for c in x)      # noqa: E731  format 103
    ivec = lambda x: "".join(_i(int(c), 13) for c in x)          # noqa: E731  format 130
    out = ["1",                                                              # '(i1)'
           "".join(_i(k, 10) for k in (n_mon, n_chain, n_mon_d, n_chain_d)),  # '(4i10)'
           _i(n_cell_w[0], 10) + _i(n_cell_w[1], 10),                       # format 120
           _i(N_ORDER, 3)]                                                   # format 110
    for i in range(n):                                                       # format 113
        out.append(_i(a_type[i], 3) + "".join(_f(float(c), 13, 7) for c in r0[i]))
    out.extend(vec(v[i]) for i in range(n))
    out.extend(vec(a[i]) for i in range(n))
    out.append(vec(w["r0_twall"]))
    rx = np.asarray(w["rx_twall"], dtype=np.float64).reshape(3, N_ORDER)
    for order in range(1, N_ORDER + 1):
        out.append(vec(rx[:, order - 1] / dt ** order))
    out.append(ivec(w["pbc_twall"]))
    out.append(vec(w["r0_bwall"]))
    out.append(ivec(w["pbc_bwall"]))
    out.append(vec(w["r0_spring_twall"]))
    out.append(ivec(w["s_force_grad"]))
    with open(path, "w") as fh:
        fh.write("\n".join(out) + "\n")


def _fields(line: str, widths) -> list:
    """Fixed-width fields of a formatted Fortran record (blank = 0)."""
    out, pos = [], 0
    for w in widths:
        out.append(line[pos:pos + w].strip())
        pos += w
    return out


def read_conf(path: str, n_part: int, dt: float = 0.005) -> dict:
    """conf_old as init_config.f90:104-209 reads it: the header (n_mon and
    n_chain from the first two I10 fields of line 2, the wall unit cells, the
    predictor order), then types and positions, velocities, accelerations,
    and the moving-wall block when the file holds one."""
    with open(path) as fh:
        lines = fh.read().split("\n")
    if len(lines) < 4 + 3 * n_part:
        raise ValueError(f"{path}: {len(lines)} lines, fewer than a {n_part}-particle configuration holds")
    n_mon, n_chain, n_mon_d, n_chain_d = (int(x or 0) for x in _fields(lines[1].ljust(40), (10, 10, 10, 10)))
    cw = tuple(int(x or 0) for x in _fields(lines[2].ljust(20), (10, 10)))
    j_order = min(int(lines[3][:3].strip() or 0), N_ORDER)
    k = 4
    a_type = np.empty(n_part, dtype=np.int32)
    r0 = np.empty((n_part, 3))
    for i in range(n_part):
        f = _fields(lines[k + i].ljust(42), (3, 13, 13, 13))
        a_type[i] = int(f[0])
        r0[i] = [float(x or 0.0) for x in f[1:]]
    k += n_part
    row = lambda ln: [float(x or 0.0) for x in _fields(ln.ljust(45), (15, 15, 15))]  # noqa: E731
    vel = np.array([row(lines[k + i]) for i in range(n_part)])
    k += n_part
    acc = np.array([row(lines[k + i]) for i in range(n_part)])
    k += n_part
    out = {"n_mon": n_mon, "n_chain": n_chain, "n_mon_d": n_mon_d, "n_chain_d": n_chain_d,
           "n_cell_w": cw, "n_order": j_order, "a_type": a_type, "r0": r0, "v": vel, "a": acc}
    rest = [ln for ln in lines[k:] if ln.strip()]
    if len(rest) >= 1 + j_order + 5:
        vec = lambda ln: np.array(row(ln))  # noqa: E731
        ivec = lambda ln: np.array([int(x or 0) for x in _fields(ln.ljust(39), (13, 13, 13))])  # noqa: E731
        rx = np.zeros((3, N_ORDER))
        for order in range(1, j_order + 1):
            rx[:, order - 1] = vec(rest[order]) * dt ** order
        out["walls"] = {"r0_twall": vec(rest[0]), "rx_twall": rx, "pbc_twall": ivec(rest[1 + j_order]),
                        "r0_bwall": vec(rest[2 + j_order]), "pbc_bwall": ivec(rest[3 + j_order]),
                        "r0_spring_twall": vec(rest[4 + j_order]), "s_force_grad": ivec(rest[5 + j_order])
                        if len(rest) > 5 + j_order else np.zeros(3, int)}
    return out


def write_state(path: str, r0, v, a, mic, a_type, i_time: int, bin_type: int = 0) -> None:
    """Every bit of the dynamic state (layout in the module docstring)."""
    r0 = np.ascontiguousarray(r0, dtype="<f8").reshape(-1, 3)
    n = r0.shape[0]
    arrays = [r0, np.ascontiguousarray(v, dtype="<f8").reshape(n, 3),
              np.ascontiguousarray(a, dtype="<f8").reshape(n, 3),
              np.ascontiguousarray(mic, dtype="<i4").reshape(n, 3),
              np.ascontiguousarray(a_type, dtype="<i4").reshape(n)]
    with open(path, "wb") as fh:
        fh.write(MAGIC + struct.pack("<iiqii", VERSION, n, int(i_time), int(bin_type), 0))
        for x in arrays:
            fh.write(x.tobytes())


def read_state(path: str) -> dict:
    with open(path, "rb") as fh:
        head = fh.read(24)
        if len(head) != 24 or head[:8] != MAGIC:
            raise ValueError(f"{path}: not a state file")
        version, n, i_time = struct.unpack("<iiq", head[8:])
        bin_type = None
        if version == 2:
            bin_type, _ = struct.unpack("<ii", fh.read(8))
        elif version != 1:
            raise ValueError(f"{path}: version {version}, expected 1 or {VERSION}")
        body = fh.read()
    sizes = [24 * n, 24 * n, 24 * n, 12 * n, 4 * n]
    if len(body) != sum(sizes):
        raise ValueError(f"{path}: {len(body)} bytes of arrays, expected {sum(sizes)}")
    off, out = 0, {}
    for name, size, dt, shape in (("r0", sizes[0], "<f8", (n, 3)), ("v", sizes[1], "<f8", (n, 3)),
                                  ("a", sizes[2], "<f8", (n, 3)), ("mic", sizes[3], "<i4", (n, 3)),
                                  ("a_type", sizes[4], "<i4", (n,))):
        out[name] = np.frombuffer(body[off:off + size], dtype=dt).reshape(shape).copy()
        off += size
    out["i_time"] = i_time
    out["bin_type"] = bin_type
    return out


def save(system, conf_path: str | None = None, state_path: str | None = None, n_cell_w=(0, 0)) -> None:
    """Writes a System's state: the reference's text restart file (conf_path)
    and/or the exact side-car (state_path).  Synchronises with the device."""
    from . import _abi
    st = system.download(_abi.R0 | _abi.V | _abi.A | _abi.MIC)
    p = system.params
    if conf_path:
        write_conf(conf_path, st["r0"], st["v"], st["a"], system.a_type, p.n_mon, p.n_chain, p.n_mon_d,
                   p.n_chain_d, n_cell_w, dt=p.dt)
    if state_path:
        write_state(state_path, st["r0"], st["v"], st["a"], st["mic"], system.a_type,
                    system.scalars()["i_time"], getattr(system, "bin_type", 0))


def restore(system, state_path: str | None = None, conf_path: str | None = None) -> None:
    """Loads a saved state into a System with the same particles: every bit from
    the side-car (and its step counter), or the text file's 7 decimals (step
    counter left as it is).  Then rebuilds the cells and neighbour lists from
    the loaded positions with the system's own list rule (binning or
    my_binning; a side-car written from a system of the other rule is
    refused), as the reference's start-up does after reading conf_old with the
    rule it was built with (init_config.f90:251-255)."""
    if (state_path is None) == (conf_path is None):
        raise ValueError("give exactly one of state_path and conf_path")
    if state_path:
        st = read_state(state_path)
        if st["r0"].shape[0] != system.n or (st["a_type"] != system.a_type).any():
            raise ValueError(f"{state_path}: particles differ from the system's")
        rule = getattr(system, "bin_type", 0)
        if st["bin_type"] is not None and st["bin_type"] != rule:
            raise ValueError(f"{state_path}: saved with list rule {st['bin_type']}, the system uses {rule}")
        system.upload(r0=st["r0"], v=st["v"], a=st["a"], mic=st["mic"])
        system.set_step(st["i_time"])
    else:
        st = read_conf(conf_path, system.n, dt=system.params.dt)
        if (st["a_type"] != system.a_type).any():
            raise ValueError(f"{conf_path}: particle types differ from the system's")
        system.upload(r0=st["r0"], v=st["v"], a=st["a"])
    if hasattr(system, "rebuild"):
        system.rebuild()
    else:
        system.binning()
