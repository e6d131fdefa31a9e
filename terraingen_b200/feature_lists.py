"""Crater lists as the reference writes them (WriteCraterList, src/io/feature_lists.cpp:395-409).

The columns come straight from the arrays a population hands over (tg_crater_generate's x, y,
diameter, age and id, host arrays or CUDA tensors): CSV with a header row, doubles as `%.17g`,
ids as integers and the flags as 1 or 0 (CsvText, feature_lists.cpp:84); or JSON, an object
{"craters": [...]} of one object per crater keyed by column in order, indented by 2 (CraterJson
dumped with indent 2), NaN and infinities as null. The format follows the path's extension
(".json" is JSON, anything else CSV: InferListFormat, feature_lists.cpp:27).
"""

from __future__ import annotations

import json
import math
from pathlib import Path

import numpy as np

CRATER_COLUMNS = ("x", "y", "diameter", "age_gyr", "id", "manual", "replace")


def _host(values, dtype) -> np.ndarray:
    if hasattr(values, "detach"):
        values = values.detach().cpu().numpy()
    return np.ascontiguousarray(values, dtype)


def _json_number(v: float):
    return v if math.isfinite(v) else None


def write_crater_list(path, x, y, diameter, age_gyr, ids, manual=None, replace=None,
                      format: str | None = None) -> None:
    """Writes the craters to `path`; `format` "csv" or "json" overrides the extension."""
    cols = [_host(v, np.float64) for v in (x, y, diameter, age_gyr)]
    n = len(cols[0])
    ident = _host(ids, np.uint64)
    man = np.zeros(n, bool) if manual is None else _host(manual, bool)
    rep = np.zeros(n, bool) if replace is None else _host(replace, bool)
    if any(len(c) != n for c in (*cols, ident, man, rep)):
        raise ValueError("every column needs one value per crater")
    path = Path(path)
    fmt = format or ("json" if path.suffix.lower() == ".json" else "csv")
    if fmt == "csv":
        lines = [",".join(CRATER_COLUMNS)]
        for i in range(n):
            cells = ["%.17g" % float(c[i]) for c in cols]
            cells += [str(int(ident[i])), "1" if man[i] else "0", "1" if rep[i] else "0"]
            lines.append(",".join(cells))
        path.write_text("\n".join(lines) + "\n")
    elif fmt == "json":
        rows = []
        for i in range(n):
            row = {name: _json_number(float(c[i])) for name, c in zip(CRATER_COLUMNS, cols)}
            row["id"] = int(ident[i])
            row["manual"] = bool(man[i])
            row["replace"] = bool(rep[i])
            rows.append(row)
        path.write_text(json.dumps({"craters": rows}, indent=2) + "\n")
    else:
        raise ValueError("format must be csv or json")
