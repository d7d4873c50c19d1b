"""Statistical parity on the target lattices: 32^4 at beta = 0.9, 1.0, 1.1
and 24^3 x 48 with xi = 2 (reference arguments beta = 2, aniso = 2).

Our chain (1 Metropolis + 4 OR per sweep, measured every sweep) against the
reference's own CUDA chain from the same start configuration, and, for the
32^4 beta = 1.0 configuration, against a short FP64 oracle chain started
from our thermalised configuration.  <Re P_SS>, <Re P_ST> and <|L|> agree
within 4 combined errors (the larger of the binned-jackknife and the
Gamma-method error of each chain).  The full-length runs (5000 sweeps) are
made by `python -m tests.target_parity`, which these tests share.
"""
import numpy as np
import pytest

from oracle.oracle import Ref
from tests import target_parity as tp

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not Ref.available(), reason="oracle/_ref not built (reference sources absent)")]

SWEEPS, THERM = 2000, 250


@pytest.mark.parametrize("k", range(len(tp.CONFIGS)), ids=[c["name"] for c in tp.CONFIGS])
def test_target_lattice_vs_reference_cuda(ctx, k):
    cfg = tp.CONFIGS[k]
    th0, th_therm, ours = tp.run_ours(ctx, cfg, SWEEPS, THERM)
    ref = tp.run_reference_cuda(cfg, th0, THERM + SWEEPS)
    so = tp.summarize(tp.observables(ours[THERM:]))
    sr = tp.summarize(tp.observables(ref[THERM:]))
    p = tp.pulls(so, sr)
    assert all(abs(v) < 4.0 for v in p.values()), (cfg["name"], p, so, sr)
    if cfg["beta"] == 1.0 and cfg["aniso"] == 1.0:
        orc = tp.observables(tp.run_oracle(cfg, th_therm, 40)[10:])
        sc = tp.summarize(orc, nbins=10)
        po = tp.pulls(so, sc)
        assert all(abs(v) < 4.0 for v in po.values()), (po, so, sc)
