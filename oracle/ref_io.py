"""TEST INFRASTRUCTURE: input/output files of oracle/ref_harness.cu.

Input (little endian): int64 header[16] = {magic "BESRFIN1", n_systems, units,
ndo, n_periods, reset_at, event_dir, do_save_frequency, device,
restart_each_period, 0...};
double options[16] = {dt0, dtmin, dtmax, rtol0, rtol1, atol0, atol1,
event_tol, grow, shrink, do_min_dt, 0...}; then upar [21][TU], state [2][TU],
uacc [64][TU] (double), iuacc [TU] (int32) and the N x N column-major
coupling matrix.  Output: int64 header[8] = {magic "BESRFOU1", n_systems,
units, ndo, elapsed_ns, n_periods, 0, 0}; state [2][TU], uacc [64][TU],
iuacc [TU], actual_time [NS], dense_index [NS] and, when ndo > 0,
dense_time [ndo][NS] and dense_state [ndo][2][TU]; then the seconds of each
period's Solve() + synchronisation [n_periods].
"""
from __future__ import annotations

import subprocess
from pathlib import Path

import numpy as np

MAGIC_IN = 0x4245535246494e31
MAGIC_OUT = 0x42455352464f5531


def write_input(path, ens, n_periods: int, reset_at: int, ndo: int = 0, do_min_dt: float = 0.0,
                do_save_frequency: int = 1, device: int = 0, uacc=None, iuacc=None,
                restart_each_period: bool = False) -> None:
    if len(set(ens.units.tolist())) != 1 or ens.n_matrices != 1:
        raise ValueError("the reference solver needs one unit count and one shared coupling matrix")
    ns, n = ens.n_systems, int(ens.units[0])
    hdr = np.zeros(16, np.int64)
    hdr[:10] = [MAGIC_IN, ns, n, ndo, n_periods, reset_at, ens.event_dir, do_save_frequency, device,
                int(restart_each_period)]
    opt = np.zeros(16)
    opt[:11] = [ens.dt0, ens.dtmin, ens.dtmax, ens.rtol[0, 0], ens.rtol[1, 0], ens.atol[0, 0], ens.atol[1, 0],
                ens.event_tol, ens.grow, ens.shrink, do_min_dt]
    with open(path, "wb") as f:
        f.write(hdr.tobytes())
        f.write(opt.tobytes())
        f.write(np.ascontiguousarray(ens.upar, np.float64).tobytes())
        f.write(np.ascontiguousarray(ens.state, np.float64).tobytes())
        f.write(np.ascontiguousarray(ens.initial_uacc() if uacc is None else uacc, np.float64).tobytes())
        f.write(np.ascontiguousarray((ens.initial_iuacc() if iuacc is None else iuacc).reshape(-1), np.int32).tobytes())
        f.write(np.ascontiguousarray(ens.coupling[: n * n], np.float64).tobytes())


def read_output(path) -> dict:
    raw = Path(path).read_bytes()
    hdr = np.frombuffer(raw[:64], np.int64)
    if hdr[0] != MAGIC_OUT:
        raise ValueError("bad output magic")
    ns, n, ndo = int(hdr[1]), int(hdr[2]), int(hdr[3])
    tu = ns * n
    off = 64

    def take(count, dt):
        nonlocal off
        a = np.frombuffer(raw[off: off + count * np.dtype(dt).itemsize], dt).copy()
        off += count * np.dtype(dt).itemsize
        return a

    out = {"elapsed_s": hdr[4] * 1e-9, "n_periods": int(hdr[5])}
    out["state"] = take(2 * tu, np.float64).reshape(2, tu)
    out["uacc"] = take(64 * tu, np.float64).reshape(64, tu)
    out["iuacc"] = take(tu, np.int32).reshape(1, tu)
    out["actual_time"] = take(ns, np.float64)
    out["dense_index"] = take(ns, np.int32)
    if ndo:
        out["dense_time"] = take(ndo * ns, np.float64).reshape(ndo, ns)
        out["dense_state"] = take(ndo * 2 * tu, np.float64).reshape(ndo, 2, tu)
    out["period_s"] = take(out["n_periods"], np.float64)
    return out


def run(exe, ens, n_periods: int, reset_at: int, workdir, tag: str = "run", timeout: float = 600, **kw) -> dict:
    workdir = Path(workdir)
    workdir.mkdir(parents=True, exist_ok=True)
    fin, fout = workdir / f"{tag}.in.bin", workdir / f"{tag}.out.bin"
    write_input(fin, ens, n_periods, reset_at, **kw)
    res = subprocess.run([str(exe), str(fin), str(fout)], capture_output=True, text=True, timeout=timeout)
    if res.returncode != 0:
        raise RuntimeError(f"{exe} failed ({res.returncode}):\n{res.stdout[-2000:]}\n{res.stderr[-2000:]}")
    return read_output(fout)
