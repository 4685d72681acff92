"""Split-precision Legendre stages from the precomputed INT8 digit table
(option 4 = digits, option 8 = 0; sht_ptab.cu) against the FP64 transform on
the same plan and inputs, and against the reference library.

Products of digits are summed exactly in INT32, so the error comes from the
NS digits per operand (about 8 NS - 2 bits, relative to the row and column
maxima).  Bounds are relative to the largest output value:
  * synthesis and analysis per digit count at lmax 127, 8 fields (the
    tensor-core tile of 32 columns);
  * vector (qst, several column tiles) and truncated (ltr) forms;
  * polar threshold, 64 fields of the lmax 511 grid against the FP64 stages
    and two of them against the reference library;
  * lmax 4095 (extended-exponent rows, polar threshold 1e-10), 8 fields with
    7 digits: synthesis and analysis within 1e-11 of the FP64 stages.
"""
import numpy as np
import pytest

from tests.common import rand_spec

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

# about 8x the measured errors; the leading digit keeps 6 bits plus sign
# (values scaled below 1/4 so that it fits INT8), so each digit count is
# about 4x less accurate than the same count of FP16 slices
BOUND = {3: 6e-4, 4: 3e-6, 5: 1.2e-8, 6: 5e-11, 7: 2e-13}


def _plan(L, nlat=None, eps=0.0):
    import shtns_b200
    nl = nlat or (3 * (L + 1) // 2 + (3 * (L + 1) // 2) % 2)
    sh = shtns_b200.sht(L)
    sh.set_grid(nl, 2 * nl, flags=shtns_b200.sht_quick_init | shtns_b200.SHT_THETA_CONTIGUOUS, polar_opt=eps)
    return sh


def _rel(a, b):
    return float((a - b).abs().max() / b.abs().max())


def test_table_accuracy_per_digits():
    dev = torch.device("cuda:0")
    sh = _plan(127)
    q = torch.from_numpy(rand_spec(127, 127, 1, 7, power=1.0, nfields=8)).to(dev)
    v64 = sh.synth(q)
    q64 = sh.analys(v64)
    es, ea = {}, {}
    for ns in (3, 4, 5, 6, 7):
        sh.set_split(ns)
        es[ns] = _rel(sh.synth(q), v64)
        ea[ns] = _rel(sh.analys(v64), q64)
        assert sh.kernel_errors() == 0
    print("synthesis", es, "analysis", ea)
    for ns in es:
        assert es[ns] < BOUND[ns] and ea[ns] < BOUND[ns], (es, ea)
    assert es[3] > es[5] > es[7] and ea[3] > ea[5] > ea[7]
    sh.set_split(0)
    assert torch.equal(sh.synth(q), v64)


def test_table_vector_and_truncated():
    dev = torch.device("cuda:0")
    L = 127
    sh = _plan(L)
    q = torch.from_numpy(rand_spec(L, L, 1, 11, power=1.0, nfields=3)).to(dev)
    s = torch.from_numpy(rand_spec(L, L, 1, 12, power=1.5, zero_l0=True, nfields=3)).to(dev)
    t = torch.from_numpy(rand_spec(L, L, 1, 13, power=1.5, zero_l0=True, nfields=3)).to(dev)
    ref = sh.synth(q, s, t)
    ref_a = sh.analys(*ref)
    ref_l = sh.synth(q, ltr=100)
    ref_al = sh.analys(ref_l, ltr=100)
    sh.set_split(7)
    out = sh.synth(q, s, t)
    out_a = sh.analys(*ref)
    out_l = sh.synth(q, ltr=100)
    out_al = sh.analys(ref_l, ltr=100)
    assert sh.kernel_errors() == 0
    for a, b in zip(out, ref):
        assert _rel(a, b) < 1e-13
    for a, b in zip(out_a, ref_a):
        assert _rel(a, b) < 1e-13
    assert _rel(out_l, ref_l) < 1e-13
    assert _rel(out_al, ref_al) < 1e-13


def test_table_polar_threshold_64_fields_and_reference():
    from oracle import shtns_ref as R
    dev = torch.device("cuda:0")
    L = 511
    sh = _plan(L, nlat=768, eps=1e-10)
    qn = rand_spec(L, L, 1, 21, power=1.0, nfields=64)
    q = torch.from_numpy(qn).to(dev)
    v64 = sh.synth(q)
    q64 = sh.analys(v64)
    sh.set_split(7)
    v = sh.synth(q)
    qa = sh.analys(v64)
    assert sh.kernel_errors() == 0
    assert _rel(v, v64) < 1e-12
    assert _rel(qa, q64) < 1e-12
    if R.available():
        ref = R.RefSHT(L, L, 1, R.sht_orthonormal, 768, 1536, flags=R.sht_quick_init | R.SHT_THETA_CONTIGUOUS,
                       eps=1e-10)
        for f in (0, 37):
            rv = ref.synth(qn[f])
            # polar rows: the reference rounds its first kept row to its SIMD width
            assert np.abs(v[f].cpu().numpy() - rv).max() / np.abs(rv).max() < 1e-9
            rq = ref.analys(rv)
            got = sh.analys(torch.from_numpy(rv).to(dev)).cpu().numpy()
            assert np.abs(got - rq).max() / np.abs(rq).max() < 1e-9
        ref.close()


def test_table_high_degree_within_1e11():
    dev = torch.device("cuda:0")
    L = 4095
    sh = _plan(L, nlat=6144, eps=1e-10)
    q = torch.from_numpy(rand_spec(L, L, 1, 15, power=1.0, nfields=8)).to(dev)
    v64 = sh.synth(q)
    q64 = sh.analys(v64)
    sh.set_split(7)
    v = sh.synth(q)
    qa = sh.analys(v64)
    assert sh.kernel_errors() == 0
    es, ea = _rel(v, v64), _rel(qa, q64)
    print("lmax 4095, 7 digits: synthesis", es, "analysis", ea)
    assert es < 1e-11, es
    assert ea < 1e-11, ea


def test_table_two_column_tiles_per_item():
    """Each analysis work item reads the table once for two 32-column tiles
    (accumulators of both in tensor memory), here at lmax 2047.  20 fields = 80
    GEMM columns = 3 tiles: items hold a pair of tiles or the last single one.
    Synthesis and analysis within 1e-11 of the FP64 stages, as in the 8-field
    (one tile per item) case above."""
    dev = torch.device("cuda:0")
    L = 2047
    sh = _plan(L, nlat=3072, eps=1e-10)
    q = torch.from_numpy(rand_spec(L, L, 1, 16, power=1.0, nfields=20)).to(dev)
    v64 = sh.synth(q)
    q64 = sh.analys(v64)
    sh.set_split(7)
    v = sh.synth(q)
    qa = sh.analys(v64)
    assert sh.kernel_errors() == 0
    es, ea = _rel(v, v64), _rel(qa, q64)
    print("lmax 2047, 20 fields, 7 digits: synthesis", es, "analysis", ea)
    assert es < 1e-11, es
    assert ea < 1e-11, ea
    # every field, not only the largest values: per-field errors against each field's maximum
    for f in (0, 9, 19):
        assert _rel(v[f], v64[f]) < 1e-11
        assert _rel(qa[f], q64[f]) < 1e-11
