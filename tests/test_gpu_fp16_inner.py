"""Ruiz-scaled fp16 values in the GMRES-IR inner products (inner_prec 2):
used only where every scaled nonzero lies in the fp16 normal range, decided
per system on the device; the answer is the fp64 oracle's either way."""
import numpy as np
import pytest

from luspice_b200 import api, mna
from tests.helpers import TOL_REL, oracle_solution, rel_err, rel_res, ruiz_fits_fp16

pytestmark = pytest.mark.gpu

@pytest.mark.parametrize("case", ["grid", "analog"])
def test_fp16_inner_products_where_they_fit(gpu, case):
    m = mna.power_grid() if case == "grid" else mna.analog(989, 42)
    P = api.Pattern.from_matrix(m)
    vals = m.perturbed(4, seed=13)
    fits = [ruiz_fits_fp16(m, v) for v in vals]
    # fp16 inner products gain about three digits per outer step: room for more.
    B = api.Batch([P] * 4, prec=api.MIXED, inner_prec=api.INNER_FP16, max_outer=8)
    B.upload(list(vals), [m.b] * 4)
    B.run(api.RUN_BOTH)
    xs = B.split(B.download())
    st = B.stats()
    _, q = P.perm()
    for s in range(4):
        assert bool(st[s]["status"] & api.ST_FP16_OFF) == (not fits[s]), (fits[s], st[s]["status"])
        assert st[s]["status"] & api.ST_FAIL_MASK == 0, st[s]
        assert rel_err(xs[s], oracle_solution(m, vals[s], q=q)) <= TOL_REL
        assert rel_res(m, vals[s], xs[s], m.b) <= 1e-9
        assert st[s]["res"][-1] <= 1e-10
    if case == "grid":
        assert all(fits)        # conductances within 2 decades: fp16 is used
    else:
        assert not any(fits)    # gmin 1e-12 next to 1e-1 conductances: fp32


def test_fp16_refused_when_range_does_not_fit(gpu):
    """Values spread over 15 decades: equilibration cannot bring them into
    the fp16 normal range, the device says so and runs the fp32 inner
    products instead: the same answer, bit for bit, as inner_prec 0."""
    m = mna.large_circuit(3000, seed=5)
    assert m.meta["frac_below_fp16_normal"] > 0.04
    assert not ruiz_fits_fp16(m, m.Ax)
    P = api.Pattern.from_matrix(m)
    xs, st = {}, {}
    for ip in (api.INNER_FP32, api.INNER_FP16):
        B = api.Batch([P], prec=api.MIXED, inner_prec=ip, max_outer=6)
        B.upload([m.Ax], [m.b])
        B.run(api.RUN_BOTH)
        xs[ip] = B.download()
        st[ip] = B.stats()[0]
    assert st[api.INNER_FP16]["status"] & api.ST_FP16_OFF
    assert not st[api.INNER_FP32]["status"] & api.ST_FP16_OFF
    assert np.array_equal(xs[api.INNER_FP16].view(np.uint64), xs[api.INNER_FP32].view(np.uint64))
    assert st[api.INNER_FP16]["status"] & ~api.ST_FP16_OFF == st[api.INNER_FP32]["status"]
    assert st[api.INNER_FP16]["res"] == st[api.INNER_FP32]["res"]


def test_fp16_same_answer_class_as_fp32(gpu):
    """fp16 and fp32 inner products reach the same fp64-accurate answer (the
    outer residual is fp64 either way)."""
    m = mna.power_grid(15, 16, 6, seed=3)
    P = api.Pattern.from_matrix(m)
    vals = m.perturbed(2, seed=1)
    assert all(ruiz_fits_fp16(m, v) for v in vals)
    out = {}
    for ip in (api.INNER_FP32, api.INNER_FP16):
        B = api.Batch([P] * 2, prec=api.MIXED, inner_prec=ip, max_outer=8)
        B.upload(list(vals), [m.b] * 2)
        B.run(api.RUN_BOTH)
        out[ip] = B.split(B.download())
        assert not any(s["status"] & api.ST_FP16_OFF for s in B.stats())
    for s in range(2):
        assert rel_err(out[api.INNER_FP16][s], out[api.INNER_FP32][s]) <= 1e-9
