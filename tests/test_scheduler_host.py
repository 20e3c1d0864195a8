"""Scheduler configuration on the host: RenderProcessScheduler keys and
SetTerminationMode (sched.h:85, sched.mt.cpp:68-90)."""
import pytest

from lightmetrica_b200 import create_scheduler


def test_configuration_and_termination_mode():
    s = create_scheduler("mt")
    s.configure({"num_samples": 1024, "progress_image_interval": 0.5})
    assert s.num_samples == 1024 and s.progress_image_interval == 0.5
    assert s.termination_mode == "samples"
    s.set_termination_mode("time", 1.5)
    assert (s.termination_mode, s.termination_time) == ("time", 1.5)
    s.set_termination_mode("samples")
    assert s.termination_mode == "samples"
    with pytest.raises(ValueError):
        s.set_termination_mode("time", 0)
    with pytest.raises(ValueError):
        s.set_termination_mode("frames", 1)
    with pytest.raises(ValueError):
        s.configure({"num_samples": 0})
