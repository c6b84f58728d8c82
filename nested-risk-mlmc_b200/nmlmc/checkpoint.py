"""Reader of the MLMC driver's checkpoint file (nmlmc_mlmc_run_ckpt / nmlmc_mlmc_run_cb_ckpt).

Layout (little-endian): b"NMLMCCK1", u32 version (1), u32 bytes of the fixed part; the input
parameters targetTOL, startTOL, theta, starting_level_coeff, Ca (f64) and M0 (u64); the iteration
state: next iteration, total iterations, number of levels, starting level (u32), sample_level
calls (u64), TOL, bias_est, stat_error, elapsed seconds (f64); per level M (u64), the sums of
phi_f^k and (phi_f - phi_c)^k for k = 1..4, work and time (f64); the sampler state (u64 size and
bytes).
"""
import struct

import numpy as np

MAGIC = b"NMLMCCK1"


def read_checkpoint(path) -> dict:
    """The checkpoint's fields; ValueError for anything that is not a complete checkpoint."""
    with open(path, "rb") as f:
        b = f.read()
    try:
        return _parse(b, path)
    except struct.error as e:          # shorter than its own layout says
        raise ValueError(f"{path}: truncated checkpoint ({e})") from None


def _parse(b: bytes, path) -> dict:
    if b[:8] != MAGIC:
        raise ValueError(f"{path}: not an nmlmc checkpoint")
    version, fixed = struct.unpack_from("<II", b, 8)
    if version != 1:
        raise ValueError(f"{path}: checkpoint version {version}")
    o = 16
    targetTOL, startTOL, theta, coeff, Ca, M0 = struct.unpack_from("<5dQ", b, o)
    o += 48
    itr_next, total_itrs, nlev, starting_level, calls = struct.unpack_from("<4IQ", b, o)
    o += 24
    TOL, bias_est, stat_error, elapsed = struct.unpack_from("<4d", b, o)
    o += 32
    if o != fixed:
        raise ValueError(f"{path}: fixed part of {fixed} bytes, expected {o}")
    rec = np.dtype([("M", "<u8"), ("fsums", "<f8", 4), ("diffsums", "<f8", 4), ("work", "<f8"),
                    ("time", "<f8")])
    if not 0 < nlev <= 64 or o + nlev * rec.itemsize > len(b):
        raise ValueError(f"{path}: {nlev} levels do not fit the file")
    levels = np.frombuffer(b, rec, count=nlev, offset=o)
    o += nlev * rec.itemsize
    (ns,) = struct.unpack_from("<Q", b, o)
    o += 8
    if o + ns != len(b):
        raise ValueError(f"{path}: truncated sampler state")
    return dict(targetTOL=targetTOL, startTOL=startTOL, theta=theta, starting_level_coeff=coeff, Ca=Ca,
                M0=M0, itr_next=itr_next, total_itrs=total_itrs, starting_level=starting_level,
                calls=calls, TOL=TOL, bias_est=bias_est, stat_error=stat_error, elapsed=elapsed,
                level_M=levels["M"].copy(), level_fsums=levels["fsums"].copy(),
                level_diffsums=levels["diffsums"].copy(), level_work=levels["work"].copy(),
                level_time=levels["time"].copy(), sampler_state=b[o:o + ns])
