"""The transient waveforms (pytcad/transient.py:45-106 restated)."""
import pytest

from tcad_b200.transient import (ConstantWaveform, PulseWaveform, RampWaveform,
                                 StepWaveform, as_waveform)


def test_waveform_values():
    s = StepWaveform(0.0, 0.3, 1e-9)
    assert (s.value(0.0), s.value(1e-9), s.value(2e-9)) == (0.0, 0.3, 0.3)
    r = RampWaveform(0.0, 1.0, 1.0, 3.0)
    assert (r.value(0.5), r.value(2.0), r.value(4.0)) == (0.0, 0.5, 1.0)
    p = PulseWaveform(0.1, 0.9, 1.0, 2.0)
    assert (p.value(0.9), p.value(1.0), p.value(2.9), p.value(3.0)) == (0.1, 0.9, 0.9, 0.1)
    assert ConstantWaveform(0.7).value(123.0) == 0.7
    assert as_waveform(0.2).value(5.0) == 0.2 and as_waveform(s) is s


def test_waveform_arguments_checked():
    with pytest.raises(ValueError):
        RampWaveform(0.0, 1.0, 2.0, 2.0)
    with pytest.raises(ValueError):
        PulseWaveform(0.0, 1.0, 0.0, 0.0)
