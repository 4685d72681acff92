"""Split-precision Legendre synthesis on the FP16 tensor cores (option 4 with
option 8 = 1: slices regenerated on the fly; synthesis only).

Slices are 8-bit integers, so each kept product is summed exactly; the error
comes only from the NS slices per operand (about 8 NS bits, relative to the
row / column maxima) and is checked against the FP64 contraction on the same
plan and inputs:
  * accuracy per slice count at lmax 127 (bounds about 8x the measured
    errors), no kernel wait gave up;
  * identical results for every recurrence checkpoint spacing (8, 16, 32:
    the generators restart from different checkpoints, mid-segment for 32);
  * vector (qst) and truncated (ltr) synthesis;
  * lmax 4095 (extended-exponent rows, 32-step checkpoints) with 7 slices.
"""
import numpy as np
import pytest

from tests.common import rand_spec

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

BOUND = {3: 5e-5, 4: 2e-7, 5: 1e-9, 6: 5e-12, 7: 2e-14}


def _plan(L, nlat=None, eps=0.0):
    import shtns_b200
    nl = nlat or (3 * (L + 1) // 2 + (3 * (L + 1) // 2) % 2)
    sh = shtns_b200.sht(L)
    sh.set_grid(nl, 2 * nl, flags=shtns_b200.sht_quick_init | shtns_b200.SHT_THETA_CONTIGUOUS, polar_opt=eps)
    return sh


def _rel(a, b):
    return float((a - b).abs().max() / b.abs().max())


def test_split_accuracy_per_slices():
    dev = torch.device("cuda:0")
    sh = _plan(127)
    q = torch.from_numpy(rand_spec(127, 127, 1, 7, power=1.0, nfields=8)).to(dev)
    v64 = sh.synth(q)
    errs = {}
    for ns in (3, 4, 5, 6, 7):
        sh.set_split(ns, form=1)
        errs[ns] = _rel(sh.synth(q), v64)
        assert errs[ns] < BOUND[ns], (ns, errs[ns])
        assert sh.kernel_errors() == 0
    assert errs[3] > errs[4] > errs[5] > errs[6] > errs[7]
    sh.set_split(0)
    assert torch.equal(sh.synth(q), v64)


@pytest.mark.parametrize("ns", [5, 7])
def test_split_checkpoint_spacings_agree(ns):
    from shtns_b200 import capi
    lib = capi.load()
    dev = torch.device("cuda:0")
    sh = _plan(255)
    q = torch.from_numpy(rand_spec(255, 255, 1, 9, power=1.0, nfields=4)).to(dev)
    v64 = sh.synth(q)
    sh.set_split(ns, form=1)
    outs = []
    for seg in (8, 16, 32):
        assert lib.shtns_b200_set_option(sh._cfg, 2, seg) == 0
        outs.append(sh.synth(q))
    assert sh.kernel_errors() == 0
    assert torch.equal(outs[0], outs[1]) and torch.equal(outs[0], outs[2])
    assert _rel(outs[0], v64) < BOUND[ns] * 4


def test_split_vector_and_truncated():
    dev = torch.device("cuda:0")
    L = 127
    sh = _plan(L)
    q = torch.from_numpy(rand_spec(L, L, 1, 11, power=1.0, nfields=3)).to(dev)
    s = torch.from_numpy(rand_spec(L, L, 1, 12, power=1.5, zero_l0=True, nfields=3)).to(dev)
    t = torch.from_numpy(rand_spec(L, L, 1, 13, power=1.5, zero_l0=True, nfields=3)).to(dev)
    ref = sh.synth(q, s, t)
    ref_l = sh.synth(q, ltr=100)
    sh.set_split(7, form=1)
    out = sh.synth(q, s, t)
    out_l = sh.synth(q, ltr=100)
    assert sh.kernel_errors() == 0
    for a, b in zip(out, ref):
        assert _rel(a, b) < 1e-13
    assert _rel(out_l, ref_l) < 1e-13


def test_split_high_degree():
    dev = torch.device("cuda:0")
    L = 4095
    sh = _plan(L, nlat=6144, eps=1e-10)
    q = torch.from_numpy(rand_spec(L, L, 1, 15, power=1.0, nfields=2)).to(dev)
    v64 = sh.synth(q)
    sh.set_split(7, form=1)
    e7 = _rel(sh.synth(q), v64)
    sh.set_split(6, form=1)
    e6 = _rel(sh.synth(q), v64)
    assert sh.kernel_errors() == 0
    assert e7 < 1e-12 and e6 < 5e-10
