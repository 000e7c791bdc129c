"""metrics.csv in the reference's format (MetricsSink::flushStageCsv, src/util/metrics.cpp:78-99).

One header line, then every stage's rows in run order. Integers are written as integers and the
other numbers as the reference's stream does with std::setprecision(10) (printf's "%.10g"); float
fields are the float values widened to double, as the stream widens them.
"""
from __future__ import annotations

import numpy as np

from . import abi

HEADER = ("stage,iter,hpwl,overflow,lambda,gamma,step_size,"
          "grad_norm_wl,grad_norm_den,max_displacement,elapsed_ms,"
          "eval_lambda,eval_gamma,delta_hpwl,lambda_mu,evaluations")

# toString(GpStage) (src/gp/eplace.cpp:25-31)
STAGE_NAMES = {abi.STAGE_MGP: "mGP", abi.STAGE_FILLER_ONLY: "FILLERONLY", abi.STAGE_CGP: "cGP"}

# the columns after `stage`, their metrics-row field and whether the reference writes an integer
COLUMNS = (("iter", "iter", True), ("hpwl", "hpwl", False), ("overflow", "overflow", False),
           ("lambda", "lambda_", False), ("gamma", "gamma", False), ("step_size", "step_size", False),
           ("grad_norm_wl", "grad_norm_wl", False), ("grad_norm_den", "grad_norm_den", False),
           ("max_displacement", "max_displacement", False), ("elapsed_ms", "elapsed_ms", False),
           ("eval_lambda", "eval_lambda", False), ("eval_gamma", "eval_gamma", False),
           ("delta_hpwl", "delta_hpwl", False), ("lambda_mu", "lambda_mu", False),
           ("evaluations", "evaluations", True))


def format_number(v, integer: bool) -> str:
    if integer:
        return str(int(v))
    return format(float(v), ".10g")


def csv_text(stages) -> str:
    """The file's text for `stages`: a sequence of (stage name, rows), rows as returned by
    GpContext.metrics() (a dict of per-field arrays)."""
    out = [HEADER]
    for name, rows in stages:
        n = len(rows["iter"]) if len(rows) else 0
        for i in range(n):
            out.append(",".join([name] + [format_number(rows[f][i], integer) for _, f, integer in COLUMNS]))
    return "\n".join(out) + "\n"


def write_metrics_csv(path: str, stages) -> None:
    with open(path, "w") as f:
        f.write(csv_text(stages))


def empty_rows() -> dict:
    return {f: np.zeros(0) for _, f, _ in COLUMNS}
