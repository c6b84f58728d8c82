"""Reader of the driver's printed iteration reports (the reference's mlmc_output_t::to_string text
with its table_t layout, which nmlmc_mlmc_run produces unchanged).

Each report starts with "TOL: ..." and holds "key: value" lines (TOL, RMS, Eg, Discarded Work,
Discarded Time, Total Work, Total Time) and a table with one row per level; levels below the
starting level are printed as "*ell".  The reference's own reader (parse_mlmc_output.py) fails on
such rows (it refers to an undefined name there) and runs a parse of a fixed file when imported;
this reader is a library function and records the starting level as the number of starred rows.
"""
import re

import numpy as np

_ANSI = re.compile(r"\x1b\[\d+(;\d+)*m")


def parse_reports(text: str) -> list:
    """All reports in `text` (a driver's stdout or the table it returns), in order.  Each is a
    dict: the key/value lines as floats, 'columns' (the table header after 'ell'), 'data'
    (levels x columns array), 'starting_level'."""
    reports = []
    cur = None
    for raw in text.splitlines():
        line = _ANSI.sub("", raw).strip()
        if not line or line.startswith("#") or line.startswith("+"):
            continue
        if line.startswith("|"):
            if cur is None:
                raise ValueError(f"table row before any report: {raw!r}")
            cells = [c.strip() for c in line.strip("|").split("|")]
            if cells[0] == "ell":
                cur["columns"] = cells[1:]
                continue
            starred = cells[0].startswith("*")
            ell = int(cells[0].lstrip("*"))
            if ell != len(cur["rows"]):
                raise ValueError(f"level {ell} out of order: {raw!r}")
            cur["rows"].append([float(x) for x in cells[1:]])
            if starred:
                cur["starting_level"] = ell + 1
            continue
        key, sep, rest = line.partition(":")
        if not sep:
            raise ValueError(f"unrecognised line: {raw!r}")
        key = key.strip()
        parts = rest.split()
        if not parts:
            raise ValueError(f"no value: {raw!r}")
        value = float(parts[0])
        if key == "TOL":
            cur = dict(columns=[], rows=[], starting_level=0)
            reports.append(cur)
        elif cur is None:
            raise ValueError(f"key before any report: {raw!r}")
        cur[key] = value
    for r in reports:
        r["data"] = np.array(r.pop("rows"), dtype=float).reshape(-1, len(r["columns"]))
    return reports


def column(report: dict, name: str) -> np.ndarray:
    """One table column of a report (dEl, fEl, dVl, fVl, dKl, fKl, Wl, M, Time)."""
    return report["data"][:, report["columns"].index(name)]
