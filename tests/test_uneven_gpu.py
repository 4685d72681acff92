"""Fields of uneven lmax through a plan group (one persistent Legendre launch
per direction), its CUDA-graph replay and the autotuner.

Checks, on seeded N(0,1)/(l+1) coefficients:
  * group synthesis and analysis equal the per-bucket batched cu_* transforms
    (same kernels, same arithmetic: bit-exact) and the per-field transforms;
  * synthesis agrees with the reference's CPU library to 1e-12 for fields of
    each lmax (where the reference was built) and the round trip recovers the
    coefficients to 1e-12;
  * a CUDA-graph replay reproduces the eager result bit-exactly, and replays
    again correctly after the inputs change in place;
  * every autotuned option set gives the same results to 1e-13 and the choice
    is cached.
"""
import json

import numpy as np
import pytest

from tests.common import rand_spec, relerr

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

LMAXS = (63, 127, 255)


def _make(lmaxs, seed=7, polar_opt=0.0):
    from shtns_b200 import batch as B
    ub = B.UnevenBatch(lmaxs, device="cuda:0", polar_opt=polar_opt)
    for b, (l, n) in enumerate(zip(ub.buckets, ub.count)):
        ub.Q[b].copy_(torch.from_numpy(rand_spec(l, l, 1, seed + b, power=1.0, nfields=n)))
    return ub


@pytest.fixture(scope="module")
def small():
    lm = np.random.default_rng(3).choice(LMAXS, size=24)
    return _make(lm)


def test_group_equals_per_bucket_and_per_field(small):
    ub = small
    ub.pair()
    torch.cuda.synchronize()
    V, R = [v.clone() for v in ub.V], [r.clone() for r in ub.R]
    ub.pair_per_bucket()
    torch.cuda.synchronize()
    for a, b in zip(V, ub.V):
        assert torch.equal(a, b)
    for a, b in zip(R, ub.R):
        assert torch.equal(a, b)
    ub.pair_per_field()
    torch.cuda.synchronize()
    for a, b in zip(V, ub.V):
        assert float((a - b).abs().max() / a.abs().max()) < 1e-14
    for a, b in zip(R, ub.R):
        assert float((a - b).abs().max() / a.abs().max()) < 1e-14


def test_group_against_reference_and_roundtrip(small):
    from oracle import shtns_ref as R
    ub = small
    ub.pair()
    torch.cuda.synchronize()
    for b, sh in enumerate(ub.plans):
        assert relerr(ub.Q[b].cpu().numpy(), ub.R[b].cpu().numpy()) < 1e-12
    if not R.available():
        pytest.skip("reference library not built")
    for b, sh in enumerate(ub.plans):
        ref = R.RefSHT(sh.lmax, sh.lmax, 1, R.sht_orthonormal, sh.nlat, sh.nphi,
                       flags=R.sht_quick_init | R.SHT_THETA_CONTIGUOUS, eps=0.0, nthreads=8)
        q = ub.Q[b].cpu().numpy()
        for j in range(min(3, q.shape[0])):
            v = ref.synth(q[j])
            assert relerr(v, ub.V[b][j].cpu().numpy()) < 1e-12
        ref.close()


def test_graph_replay(small):
    ub = small
    ub.pair()
    torch.cuda.synchronize()
    V, R = [v.clone() for v in ub.V], [r.clone() for r in ub.R]
    for v in ub.V:
        v.zero_()
    for r in ub.R:
        r.zero_()
    ub.capture()
    ub.replay()
    torch.cuda.synchronize()
    for a, b in zip(V, ub.V):
        assert torch.equal(a, b)
    for a, b in zip(R, ub.R):
        assert torch.equal(a, b)
    # new inputs, written in place: the replay transforms them
    Q0 = [q.clone() for q in ub.Q]
    for q in ub.Q:
        q.mul_(-2.0)
    ub.replay()
    torch.cuda.synchronize()
    for a, b in zip(V, ub.V):
        assert float((a * -2.0 - b).abs().max() / a.abs().max()) < 1e-14
    for q, r in zip(ub.Q, ub.R):
        assert relerr(q.cpu().numpy(), r.cpu().numpy()) < 1e-12
    for q, q0 in zip(ub.Q, Q0):
        q.copy_(q0)
    ub.release_graph()


@pytest.mark.parametrize("concurrent", [0, 1])
def test_group_per_plan_legendre_form(small, concurrent):
    """Group option 5 = 1 (each bucket's own Legendre kernels, chained with its
    prologue and FFT) with the side streams on or off (option 4): the same
    results as the persistent form, eagerly and replayed from a CUDA graph."""
    ub = small
    ub.group.set_option(5, 0)
    ub.pair()
    torch.cuda.synchronize()
    V, R = [v.clone() for v in ub.V], [r.clone() for r in ub.R]
    ub.group.set_option(4, concurrent)
    ub.group.set_option(5, 1)
    try:
        for v in ub.V:
            v.zero_()
        ub.pair()
        torch.cuda.synchronize()
        for a, b in zip(V, ub.V):
            assert float((a - b).abs().max() / a.abs().max()) < 1e-14
        for a, b in zip(R, ub.R):
            assert float((a - b).abs().max() / a.abs().max()) < 1e-14
        for v in ub.V:
            v.zero_()
        for r in ub.R:
            r.zero_()
        ub.capture()
        ub.replay()
        torch.cuda.synchronize()
        for a, b in zip(V, ub.V):
            assert float((a - b).abs().max() / a.abs().max()) < 1e-14
        for a, b in zip(R, ub.R):
            assert float((a - b).abs().max() / a.abs().max()) < 1e-14
        ub.release_graph()
    finally:
        ub.group.set_option(5, 0)
        ub.group.set_option(4, 1)


def test_autotune_options_agree(small, tmp_path):
    from shtns_b200 import batch as B
    ub = small
    ub.apply_options({"fft_pairs": [1] * len(ub.plans), "ckseg": 8, "order": 1, "ctas_per_sm": 2})
    ub.pair()
    torch.cuda.synchronize()
    V0, R0 = [v.clone() for v in ub.V], [r.clone() for r in ub.R]
    path = str(tmp_path / "tune.json")
    rec = B.autotune(ub, reps=1, cache=path)
    assert set(rec["options"]) == {"fft_pairs", "ckseg", "order", "ctas_per_sm"}
    assert len(rec["trials"]) == 4 * len(ub.plans) + 12
    db = json.load(open(path))
    assert len(db) == 1 and list(db.values())[0]["options"] == rec["options"]
    for seg in (8, 16, 32):
        for pairs in (1, 2, 4, 8):
            ub.apply_options({"fft_pairs": [pairs] * len(ub.plans), "ckseg": seg, "order": 0, "ctas_per_sm": 3})
            ub.pair()
            torch.cuda.synchronize()
            for a, b in zip(V0, ub.V):
                assert float((a - b).abs().max() / a.abs().max()) < 1e-13
            for a, b in zip(R0, ub.R):
                assert float((a - b).abs().max() / a.abs().max()) < 1e-13
    # cached choice is applied without timing
    rec2 = B.autotune(ub, cache=path)
    assert rec2["options"] == rec["options"] and ub.options == rec["options"]


def test_uneven_full_workload_roundtrip():
    """256 fields, lmax uniform in {63,...,1023}: group and graph round trips."""
    lm = np.random.default_rng(2024).choice((63, 127, 255, 511, 1023), size=256)
    ub = _make(lm, seed=300)
    ub.capture()
    ub.replay()
    torch.cuda.synchronize()
    for q, r in zip(ub.Q, ub.R):
        assert relerr(q.cpu().numpy(), r.cpu().numpy()) < 1e-12
    ub.release_graph()


@pytest.mark.parametrize("kind", ["sphtor", "qst"])
@pytest.mark.parametrize("per_plan", [0, 1])
def test_group_vector_transforms_equal_plan_calls(kind, per_plan):
    """Vector fields of three lmax through one group call per direction
    (persistent Legendre launch, or each plan's own kernels with group option
    5 = 1) against each plan's own SHsphtor / SHqst calls on the same fields:
    the same arithmetic, bit-exact; one plan without fields is skipped."""
    import shtns_b200
    from shtns_b200 import batch as B
    lmaxs, counts = (47, 95, 159), (5, 0, 3)
    plans = []
    for l in lmaxs:
        nl, npn = B.grid_for(l)
        sh = shtns_b200.sht(l)
        sh.set_grid(nl, npn, flags=shtns_b200.sht_quick_init | shtns_b200.SHT_THETA_CONTIGUOUS, polar_opt=1e-10)
        plans.append(sh)
    g = B.PlanGroup(plans)
    g.set_option(5, per_plan)
    dev = torch.device("cuda:0")
    ncomp = 2 if kind == "sphtor" else 3
    spec = [[None] * 3 for _ in range(ncomp)]
    for i, (l, n) in enumerate(zip(lmaxs, counts)):
        if n == 0:
            continue
        for c in range(ncomp):
            zl0 = (ncomp == 2) or c > 0
            spec[c][i] = torch.from_numpy(rand_spec(l, l, 1, 40 + 3 * i + c, power=1.5 if zl0 else 1.0,
                                                    zero_l0=zl0, nfields=n)).to(dev)
    spat = [[None if counts[i] == 0 else torch.empty((counts[i],) + plans[i].spat_shape, dtype=torch.float64, device=dev)
             for i in range(3)] for _ in range(ncomp)]
    g.vector_synth_into(spec, spat)
    back = [[None if counts[i] == 0 else torch.empty_like(spec[c][i]) for i in range(3)] for c in range(ncomp)]
    g.vector_analys_into(spat, back)
    torch.cuda.synchronize()
    for i, sh in enumerate(plans):
        if counts[i] == 0:
            continue
        ref = sh.synth(*[spec[c][i] for c in range(ncomp)])
        for c in range(ncomp):
            assert torch.equal(ref[c], spat[c][i])
        ref_a = sh.analys(*ref)
        for c in range(ncomp):
            assert torch.equal(ref_a[c], back[c][i])
            # and the round trip recovers the input
            assert float((back[c][i] - spec[c][i]).abs().max() / spec[c][i].abs().max()) < 1e-11
    g.close()
