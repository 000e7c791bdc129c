"""metrics.csv in the reference's format (MetricsSink::flushStageCsv, src/util/metrics.cpp:78-99),
on CPU: the header, the stage order, integer columns, and the number format of a C++ stream at
std::setprecision(10), checked against the C library's own "%.10g"."""
import ctypes

import numpy as np

from superplace_b200 import abi, metrics


def c_format(v: float) -> str:
    buf = ctypes.create_string_buffer(64)
    ctypes.CDLL(None).snprintf(buf, 64, b"%.10g", ctypes.c_double(v))
    return buf.value.decode()


def rows(n, seed):
    rng = np.random.default_rng(seed)
    r = {"iter": np.arange(n), "evaluations": np.arange(n) * 2 + 3}
    for _, f, integer in metrics.COLUMNS:
        if not integer:
            r[f] = rng.standard_normal(n) * 10.0 ** rng.integers(-6, 9, n)
    r["overflow"] = r["overflow"].astype(np.float32)  # float fields are widened as the stream does
    r["max_displacement"] = np.zeros(n, np.float32)
    return r


def test_header_matches_the_reference():
    assert metrics.HEADER == ("stage,iter,hpwl,overflow,lambda,gamma,step_size,grad_norm_wl,"
                              "grad_norm_den,max_displacement,elapsed_ms,eval_lambda,eval_gamma,"
                              "delta_hpwl,lambda_mu,evaluations")


def test_rows_in_stage_order_with_the_stream_number_format():
    a, b = rows(5, 1), rows(3, 2)
    text = metrics.csv_text([("mGP", a), ("FILLERONLY", b)])
    lines = text.splitlines()
    assert lines[0] == metrics.HEADER and len(lines) == 1 + 5 + 3
    assert [ln.split(",")[0] for ln in lines[1:]] == ["mGP"] * 5 + ["FILLERONLY"] * 3
    for ln, (r, i) in zip(lines[1:], [(a, i) for i in range(5)] + [(b, i) for i in range(3)]):
        fields = ln.split(",")[1:]
        for (name, f, integer), s in zip(metrics.COLUMNS, fields):
            want = str(int(r[f][i])) if integer else c_format(float(r[f][i]))
            assert s == want, (name, s, want)


def test_special_values_and_stage_names():
    assert metrics.format_number(float("inf"), False) == c_format(float("inf"))
    assert metrics.format_number(1e10, False) == c_format(1e10) == "1e+10"
    assert metrics.format_number(0.0001234567891234, False) == c_format(0.0001234567891234)
    assert metrics.STAGE_NAMES[abi.STAGE_MGP] == "mGP"
    assert metrics.STAGE_NAMES[abi.STAGE_FILLER_ONLY] == "FILLERONLY"
    assert metrics.STAGE_NAMES[abi.STAGE_CGP] == "cGP"
