"""Plan variants of a CSR matrix (sparsep_opts.autotune).

sparsep_plan_autotune_csr_<t> times every applicable variant; a plan built
with autotune = 2 is the fastest one, with autotune = 1 the learned
selector's pick (or, at low confidence, the fastest).  Whatever the choice,
y must be the oracle's: integers bit for bit, FP32 within the per-row gamma
bound.  The block formats are offered only where blocks would be at least a
quarter full."""
import numpy as np
import pytest

import sparsep_b200 as sp
from sparsep_b200 import capi, plan_selector, synth
from helpers import fp_bound_ok, hi_ref, oracle_spmv

pytestmark = pytest.mark.gpu


def family_matrix(dtype, family, seed):
    rng = np.random.default_rng(seed)
    n, rp, ci = synth.selector_matrix(rng, family, 60_000, 12.0)
    v = (rng.uniform(-1, 1, ci.size) if dtype == "f32" else rng.integers(-8, 9, ci.size)).astype(
        capi.DTYPES[dtype].np)
    x = (rng.uniform(-1, 1, n) if dtype == "f32" else rng.integers(-8, 9, n)).astype(capi.DTYPES[dtype].np)
    return sp.csr(dtype, n, n, rp, ci, v), (rp, ci, v), x


def check(A, arrays, x, y, label):
    rp, ci, v = arrays
    n = int(A.s.nrows)
    if A.dtype == "f32":
        r = np.repeat(np.arange(n, dtype=np.uint32), np.diff(rp.astype(np.int64)))
        y_hi, a, cnt = hi_ref(r, ci, v.astype(np.float64), x.astype(np.float64), n)
        ok, err, bound = fp_bound_ok(y, y_hi, a, cnt, "f32")
        assert ok, (label, np.nonzero(err > bound)[0][:5])
    else:
        assert np.array_equal(y, oracle_spmv(A, x)), label


@pytest.mark.parametrize("dtype", ["f32", "i32"])
@pytest.mark.parametrize("family", ["uniform", "banded", "blockdiag", "rmat"])
def test_autotune_times_and_choices(dtype, family):
    A, arrays, x = family_matrix(dtype, family, seed=len(family))
    times, best = plan_selector.autotune_times(A, reps=2)
    names = plan_selector.variant_names()
    assert times[0] > 0 and times[4] > 0, "CSR and COO always apply"
    assert best == int(np.argmin(np.where(times > 0, times, np.inf)))
    print(family, dtype, {names[i]: round(float(t), 1) for i, t in enumerate(times) if t > 0})
    for mode, tag in ((2, "(autotuned)"), (1, "")):
        plan = sp.Plan(A, sp.default_opts(autotune=mode))
        variant = plan.info.variant.decode()
        assert variant.split(" ")[0] in names and tag in variant, variant
        check(A, arrays, x, plan.run_host(x), f"{family} autotune={mode} {variant}")
        plan.free()


def test_autotune_rejects_what_it_does_not_cover():
    A, _, _ = family_matrix("f32", "uniform", seed=1)
    for o in (dict(autotune=3), dict(autotune=-1)):
        with pytest.raises(capi.SparsepError) as e:
            sp.Plan(A, sp.default_opts(**o))
        assert e.value.status == capi.EINVAL
    with pytest.raises(capi.SparsepError) as e:
        sp.Plan(A, sp.default_opts(autotune=2, nrhs=4))
    assert e.value.status == capi.ENOSYS
    E = sp.cooe("f32", 10, 10, np.array([1], np.uint32), np.array([2], np.uint32), np.array([1.0], np.float32))
    with pytest.raises(capi.SparsepError) as e:
        sp.Plan(E, sp.default_opts(autotune=2))
    assert e.value.status == capi.ENOSYS


def test_learned_choice_on_held_out_matrices():
    """The plan-variant network (the library's MLP kernels, the committed
    model) against the exhaustive best on the 120 held-out matrices of the
    timing database: at most 10 % slower in total, and faster than fixed CSR."""
    from sparsep_b200 import selector

    z = np.load(plan_selector.DATA / "plan_model.npz")
    h = np.load(plan_selector.DATA / "plan_heldout.npz")
    sel = selector.selector(dict(wb=z["wb"], mean=z["mean"], std=z["std"]))
    ev = plan_selector.evaluate(sel.scores(h["feats"]), h["times"])
    print(ev)
    assert ev["samples"] == 120
    assert ev["regret_total"] <= 0.10
    assert ev["speedup_vs_fixed_csr"] > 1.0


def test_learned_choice_is_taken_when_confident():
    """With the model compiled in, autotune = 1 takes the network's pick on a
    matrix family it has seen (no timing run), and the result holds."""
    A, arrays, x = family_matrix("i32", "banded", seed=9)
    plan = sp.Plan(A, sp.default_opts(autotune=1))
    variant = plan.info.variant.decode()
    print(variant)
    assert variant.endswith("(learned)") or variant.endswith("(autotuned)")
    check(A, arrays, x, plan.run_host(x), variant)
    plan.free()
