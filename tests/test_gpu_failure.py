"""Failure detection on the GPU, without faulting, trapping or hanging it.

* A device-side wait that runs out: every mbarrier wait in the library is
  bounded by the context's wait budget (default 2 s of the GPU's global timer).
  rijk_ctx_selftest_timeout runs one such wait on a barrier that nothing
  completes (one CTA, no copy in flight); the call must return
  RIJK_ERR_TIMEOUT and the context must still give oracle-exact J and K.
* Non-finite inputs: a NaN or Inf in a density, orbital or occupation element
  that a build reads is flagged on the device and returned as
  RIJK_ERR_NONFINITE by the synchronising call; the context stays usable.

REST's own failure handling on this path is the singular-DIIS fallback
(scf_io/mod.rs:3061-3078), restated and tested in the SCF drivers.
"""
import numpy as np
import pytest

from oracle import rijk_oracle as O
from rest_b200 import RijkError
from rest_b200.synth import host_case

pytestmark = pytest.mark.gpu

TOL = 1e-10
TIMEOUT, NONFINITE, ARG = 5, 7, 1


def _maxdiff(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))))


def _still_exact(ctx, n=37, naux=150, nocc=6):
    case = host_case(n, naux, nocc, seed=41)
    ctx.set_rimatr(case.rimatr, n)
    j = ctx.vj_upper_with_rimatr_v([case.dm], 1, 1.0)[0]
    assert _maxdiff(j, O.vj_upper_with_rimatr_v(case.rimatr, [case.dm], 1, 1.0)[0]) <= TOL
    occ = np.full(nocc, 2.0)
    k = ctx.vk_upper_with_ri_v([case.c_occ], [nocc - 1], [occ], 1, -0.5)[0]
    ri3 = O.ri3fn_from_rimatr(case.rimatr, n)
    assert _maxdiff(k, O.vk_upper_with_ri_v(ri3, [case.c_occ], [nocc - 1], [occ], 1, -0.5)[0]) <= TOL


def test_wait_that_runs_out_returns_timeout_and_context_stays_usable(ctx):
    import time

    try:
        ctx.set_wait_budget(20_000_000)  # 20 ms
        t0 = time.perf_counter()
        with pytest.raises(RijkError) as ei:
            ctx.selftest_timeout()
        assert ei.value.status == TIMEOUT
        assert time.perf_counter() - t0 < 5.0
        # the flag was cleared by the call that reported it
        _still_exact(ctx)
    finally:
        ctx.set_wait_budget(0)
    # the default budget (2 s) behaves the same way
    with pytest.raises(RijkError) as ei:
        ctx.selftest_timeout()
    assert ei.value.status == TIMEOUT
    _still_exact(ctx)


def test_wait_budget_outside_its_range_is_rejected(ctx):
    for bad in (1, 9_999_999, 700 * 10**9, -5):
        with pytest.raises(RijkError) as ei:
            ctx.set_wait_budget(bad)
        assert ei.value.status == ARG


@pytest.mark.parametrize("bad", [np.nan, np.inf, -np.inf])
def test_nonfinite_density_is_reported(ctx, bad):
    n, naux, nocc = 37, 150, 6
    case = host_case(n, naux, nocc, seed=43)
    ctx.set_rimatr(case.rimatr, n)
    d = case.dm.copy(order="F")
    d[3, 20] = bad  # upper triangle: read by both J formulas and by the dm-form K
    for call in (lambda: ctx.vj_upper_with_rimatr_v([d], 1, 1.0),
                 lambda: ctx.vj_upper_with_ri_v([d], 1, 1.0),
                 lambda: ctx.vk_upper_with_rimatr_use_dm_only([d], 1, -0.5),
                 lambda: ctx.vk_full_fromdm_with_ri_v([d], 1, 1.0)):
        with pytest.raises(RijkError) as ei:
            call()
        assert ei.value.status == NONFINITE
    # a second spin with the bad value, the first clean
    with pytest.raises(RijkError) as ei:
        ctx.vj_upper_with_rimatr_v([case.dm, d], 2, 1.0)
    assert ei.value.status == NONFINITE
    _still_exact(ctx)


def test_nonfinite_orbitals_or_occupations_are_reported(ctx):
    n, naux, nocc = 37, 150, 6
    case = host_case(n, naux, nocc, seed=44)
    ctx.set_rimatr(case.rimatr, n)
    c = case.c_occ.copy(order="F")
    c[11, 2] = np.nan
    with pytest.raises(RijkError) as ei:
        ctx.vk_upper_with_ri_v([c], [nocc - 1], [np.full(nocc, 2.0)], 1, -0.5)
    assert ei.value.status == NONFINITE
    occ = np.full(nocc, 2.0)
    occ[4] = np.inf
    with pytest.raises(RijkError) as ei:
        ctx.vk_upper_with_ri_v([case.c_occ], [nocc - 1], [occ], 1, -0.5)
    assert ei.value.status == NONFINITE
    # an orbital beyond homo is not read: no error
    e = np.zeros((n, nocc + 1), order="F")
    e[:, :nocc] = case.c_occ
    e[0, nocc] = np.nan
    ctx.vk_upper_with_ri_v([e], [nocc - 1], [np.r_[np.full(nocc, 2.0), 0.0]], 1, -0.5)
    _still_exact(ctx)


def test_nonfinite_device_input_is_reported_at_synchronize(ctx):
    import torch

    n, naux, nocc = 37, 150, 6
    case = host_case(n, naux, nocc, seed=45)
    ctx.set_rimatr(case.rimatr, n)
    st = ctx.stream
    with torch.cuda.stream(torch.cuda.ExternalStream(st)):
        dm = torch.tensor(case.dm.T.ravel(), dtype=torch.float64, device="cuda")
        dm[5 * n + 2] = float("nan")  # column 5, row 2 (column-major): upper triangle
        out = torch.empty(n * (n + 1) // 2, dtype=torch.float64, device="cuda")
        ctx.vj_upper_dev(dm.data_ptr(), 1, 1.0, 1, out.data_ptr(), st)
        with pytest.raises(RijkError) as ei:
            ctx.synchronize(st)
        assert ei.value.status == NONFINITE
        # negative occupations reach the device form unchecked and are flagged there
        c = torch.tensor(case.c_occ.T.ravel(), dtype=torch.float64, device="cuda")
        occ = torch.full((nocc,), 2.0, dtype=torch.float64, device="cuda")
        occ[1] = -1.0
        ctx.vk_upper_occ_dev(c.data_ptr(), nocc, [nocc - 1], occ.data_ptr(), 1, -0.5, out.data_ptr(), st)
        with pytest.raises(RijkError) as ei:
            ctx.synchronize(st)
        assert ei.value.status == NONFINITE
        ctx.synchronize(st)  # cleared
    _still_exact(ctx)
