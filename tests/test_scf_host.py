"""Host logic of the SCF driver on the CPU: the mixed-phase screening threshold that
SingleSlater sets on its integral context, checked against a fake context."""
from chronusq_public_b200.aointegrals import PREC_FP64, PREC_MIXED
from chronusq_public_b200.scf import SingleSlater


class _FakeInts:
    def __init__(self, thresh):
        self.thresholdSchwartz = thresh
        self.calls = []

    def setPrecision(self, policy, cutoff=0.0):
        self.calls.append((policy, cutoff))


def _driver(thresh, mixed_threshold):
    hf = object.__new__(SingleSlater)      # no GPU: only the attributes _set_precision reads
    hf.ints = _FakeInts(thresh)
    hf.fp32_cutoff = 1e-8
    hf.mixed_threshold = mixed_threshold
    hf._base_threshold = None
    return hf


def test_mixed_phase_loosens_then_restores_the_threshold():
    hf = _driver(1e-14, 1e-11)
    assert hf._mixed_threshold_active()
    hf._set_precision(True)
    assert hf.ints.thresholdSchwartz == 1e-11 and hf.ints.calls[-1] == (PREC_MIXED, 1e-8)
    hf._set_precision(True)                 # a second call keeps the context's own threshold
    assert hf._base_threshold == 1e-14
    hf._set_precision(False)
    assert hf.ints.thresholdSchwartz == 1e-14 and hf.ints.calls[-1] == (PREC_FP64, 0.0)


def test_mixed_threshold_never_tightens_the_context():
    hf = _driver(1e-10, 1e-11)
    assert not hf._mixed_threshold_active()
    hf._set_precision(True)
    assert hf.ints.thresholdSchwartz == 1e-10
    hf._set_precision(False)
    assert hf.ints.thresholdSchwartz == 1e-10


def test_mixed_threshold_none_keeps_the_context_threshold():
    hf = _driver(1e-14, None)
    assert not hf._mixed_threshold_active()
    hf._set_precision(True)
    assert hf.ints.thresholdSchwartz == 1e-14 and hf.ints.calls[-1] == (PREC_MIXED, 1e-8)
