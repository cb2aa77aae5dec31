"""The reference's text formats (no GPU): ES25.17E3 numbers, the per-step CSV and the
DSTEP_BUILD.<S> record dump, checked on the oracle's weights and selection."""
import numpy as np

import oracle
from jkogb_b200 import gen, trace


def test_es25_format():
    assert trace.es25(1.0) == " 1.00000000000000000E+000"
    assert trace.es25(-0.0) == "-0.00000000000000000E+000"
    assert trace.es25(-2.5e-300) == "-2.49999999999999998E-300"  # the double nearest -2.5e-300
    assert trace.es25(1.7976931348623157e308) == " 1.79769313486231571E+308"
    assert trace.es25(float("nan")).strip() == "NaN" and len(trace.es25(float("nan"))) == 25
    assert all(len(trace.es25(x)) == 25 for x in (1e-320, 3.0, -7.25e12))


def test_csv_from_oracle_trace():
    Y, J = gen.gaussian(12, seed=3, n_plus=7)
    r = oracle.step_loop(Y, J, trace=True)
    lines = trace.csv_lines(r["trace"], 0.001)
    assert lines[0] == trace.CSV_HEADER
    assert len(lines) == r["info"] + 2  # the header, the steps with pivots, the closing step
    last = lines[-1].split(",")
    assert int(last[1]) == 0 and int(last[4]) == -1 and last[5].strip() == "-0.00000000000000000E+000"
    first = lines[1].split(",")
    assert int(first[0]) == 0 and float(first[2]) == 0.001 and len(first[5]) == 25


def test_build_dump_matches_oracle_order(tmp_path):
    Y, J = gen.graded(16, 1e-3, seed=4)
    w, P, Q, tt = oracle.weights(Y, J)
    n = 16
    W = np.full((n, n), np.nan)
    W[P - 1, Q - 1] = w
    W[Q - 1, P - 1] = w
    piv = oracle.select(n, w, P, Q, n // 2)
    # the record order: weight descending, then band, then p
    ws, ps, qs, bs = trace.sorted_records(W)
    assert len(ws) == int(np.sum(~np.isnan(w)))
    for k in range(len(ws) - 1):
        key0, key1 = (ws[k], bs[k], ps[k]), (ws[k + 1], bs[k + 1], ps[k + 1])
        assert key0 > key1
    name = trace.build_dump(5, W, piv, prefix=str(tmp_path / "DSTEP_BUILD"))
    assert name.endswith("DSTEP_BUILD.00000000005")
    text = open(name).read().splitlines()
    assert text[1] == '"J","W","P","Q","B"'
    sel_at = text.index('"I","J","W","P","Q","B"')
    rows = [r.split(",") for r in text[sel_at + 1:]]
    assert len(rows) == len(piv)
    # the selected records appear in increasing list position: the greedy walk's order
    js = [int(r[1]) for r in rows]
    assert js == sorted(js)
    for r, (a, c) in zip(rows, piv):
        assert (int(r[3]), int(r[4]), int(r[5])) == (a, c, c - a)
