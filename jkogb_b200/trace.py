"""Telemetry in the reference's text formats: the per-step CSV that DSTEP_LOOP writes to
stderr (src/D/dstep.F90:389-442, 560) from a `jk_trace`, and the per-step record dump of
a debug build, DSTEP_BUILD.<S> (AW_OUT, src/shared/atypes.F90:30-77; OPEN_LOG,
src/shared/utils.F90:79-96), from one build's weight matrix and the selected pivots.
"""
from __future__ import annotations

import math

import numpy as np

CSV_HEADER = '"STEP","OLDLEN","BUILDs","TRANSFs","NEWLEN","NORMF2D","TRIG","HYP"'


def es25(x: float) -> str:
    """Fortran ES25.17E3: 17 digits after the point, a three-digit exponent, width 25."""
    x = float(x)
    if math.isnan(x):
        return "NaN".rjust(25)
    if math.isinf(x):
        return ("-Inf" if x < 0 else "Inf").rjust(25)
    m, e = f"{x:.17E}".split("E")
    return f"{m}E{e[0]}{int(e[1:]):03d}".rjust(25)


def csv_lines(trace: dict, seconds_per_step: float = 0.0) -> list[str]:
    """The CSV of a traced solve (the `trace` dict of jkogb_b200.step_loop): one row per step,
    the last one the step without pivots.  The steps run on the GPU inside CUDA graphs, so
    BUILDs holds the given mean time per step and TRANSFs 0."""
    out = [CSV_HEADER]
    sl, nl, tw, tg, hy = (trace[k] for k in ("sl", "nl", "tw", "trig", "hyp"))
    for s in range(len(sl)):
        if sl[s] <= 0:
            row = (s, sl[s], seconds_per_step, 0.0, -1, -0.0, 0, 0)
        else:
            row = (s, sl[s], seconds_per_step, 0.0, nl[s], tw[s], tg[s], hy[s])
        out.append(f"{row[0]:11d},{row[1]:11d},{row[2]:12.6f},{row[3]:12.6f},{row[4]:11d},{es25(row[5])},"
                   f"{row[6]:11d},{row[7]:11d}")
    return out


def sorted_records(W: np.ndarray):
    """The finite records (w, p, q, b) of a symmetric weight matrix in the record order of
    AW_CMP (src/shared/atypes.F90:85-120): larger weight first, then larger band q - p, then
    larger p; p, q 1-based."""
    W = np.asarray(W, np.float64)
    n = W.shape[0]
    q0, p0 = np.triu_indices(n, 1)[1], np.triu_indices(n, 1)[0]
    w = W[p0, q0]
    ok = ~np.isnan(w)
    w, p, q = w[ok], p0[ok] + 1, q0[ok] + 1
    b = q - p
    wz = np.where(w == 0.0, 0.0, w)  # -0 and +0 are equal
    order = np.lexsort((-p, -b, -wz))
    return w[order], p[order], q[order], b[order]


def build_dump(step: int, W: np.ndarray, piv: np.ndarray, prefix: str = "DSTEP_BUILD") -> str:
    """Write the record dump of build `step` to prefix.<step as 11 digits>: the sorted records
    (J, W, P, Q, B) and the selected ones (I, J, W, P, Q, B), J their positions in the sorted
    list.  piv holds the step's pivots (p, q), 1-based, in selection order.  Returns the file
    name.  The timing lines (SRT:, NCP:, ALL:) carry 0, the GPU's work not being split so."""
    w, p, q, b = sorted_records(W)
    where = {(int(a), int(c)): j for j, (a, c) in enumerate(zip(p, q), start=1)}
    name = f"{prefix}.{int(step):011d}"
    with open(name, "w") as f:
        f.write(f"SRT: {0.0:12.6f} s\n")
        f.write('"J","W","P","Q","B"\n')
        for j in range(len(w)):
            f.write(f"{j + 1:11d},{es25(w[j])},{int(p[j]):11d},{int(q[j]):11d},{int(b[j]):11d}\n")
        f.write(f"NCP: {0.0:12.6f} s\n")
        f.write(f"ALL: {0.0:12.6f} s\n")
        f.write('"I","J","W","P","Q","B"\n')
        for i, (a, c) in enumerate(np.asarray(piv).reshape(-1, 2), start=1):
            j = where[(int(a), int(c))]
            f.write(f"{i:11d},{j:11d},{es25(w[j - 1])},{int(a):11d},{int(c):11d},{int(c - a):11d}\n")
    return name
