"""Output and restart on the device (pip_b200.output.run_with_output, IO_rot.f90's output
and restart): a run that writes every dtout, restarted from one of its outputs in a new
context, reaches the same final state bitwise -- FP64 and FP32-mixed (the mixed state's
FP32 pair is rebuilt exactly from the FP64 file), and FP64 with alpha_c per cell (the
field is written with every output and read back)."""
import numpy as np
import pytest

from pip_b200 import capi, ics, output
from pip_b200.params import PIP_FP64, PIP_MIXED

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision,flag_col", [(PIP_FP64, 1), (PIP_MIXED, 1), (PIP_FP64, 5)])
def test_restart_continues_the_run(gpu_lib, tmp_path, precision, flag_col):
    s, Uh, Um = ics.kelvin_helmholtz(64, 32, precision=precision, flag_col=flag_col)
    dtout, tend = 0.01, 0.04
    out = str(tmp_path / "run")
    with capi.Context(s) as c:
        c.upload(Uh, Um)
        c.prologue()
        st, last, t = output.run_with_output(c, s, out, dtout, tend)
    assert st == 0 and last == 4 and t >= tend
    final = output.read_output(output.file_stem(out, 4))
    # output k is written at the first step that reaches k*dtout (time >= get_next_output)
    for k in range(1, 5):
        tk = output.read_output(output.file_stem(out, k))["time"]
        assert k * dtout <= tk < (k + 1) * dtout
    # restart from output 2 (restart, IO_rot.f90:405-459) and run on to tend
    t2, h2, m2 = output.restart(out, 2, s)
    out2 = str(tmp_path / "restarted")
    with capi.Context(s) as c:
        c.upload(h2, m2)
        if flag_col >= 2:                            # reread_variables' "ac"
            c.set_alpha_c(output.restart_alpha_c(out, 2, s))
        c.time = t2
        st, last, t = output.run_with_output(c, s, out2, dtout, tend, nout0=2)
    again = output.read_output(output.file_stem(out2, 4))
    assert st == 0 and last == 4
    assert again["time"] == final["time"]
    for name in output.variables(s):
        assert np.array_equal(again[name], final[name]), name
