"""The tensor-core form's precision design, checked on the CPU.

tests/tc_replay.py replays the engine's arithmetic in numpy. At t = 1e5 on
the 512^2 foam patch (the hardest case: the FP32 form's normals are 3.5e-6
from FP64 there), the twiddle step by Kahan's difference of products keeps
every channel within 2e-6 of the FP64 frame, and rounding its products and
sum separately does not: the step that bounds the form's accuracy."""
import oracle as O
from oceanlib_b200 import workloads as W
from tests import tc_replay as R


def test_kahan_twiddle_step_keeps_the_late_time_frame_within_2e_6():
    desc, t = W.foam_patch_512(), 1.0e5
    ref = O.fp64_frame(desc, t)
    kahan = R.channel_errors(R.frame(desc, t, kahan=True), ref)
    three = R.channel_errors(R.frame(desc, t, kahan=False), ref)
    assert max(kahan.values()) <= 2e-6, kahan
    assert max(three.values()) > 2e-6, three
    assert kahan["normal.x"] < three["normal.x"]
