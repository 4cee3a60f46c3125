"""FC / window FCs on the tensor cores (FP32 mode, model_config "fc" = "tc")
against the FP64 FC kernels on the same BOLD: the Gram product of the
normalised BOLD columns in BF16x3 with FP32 accumulation must stay within 1e-4
of the FP64 Pearson r (its error is about 1e-5), the FCD computed from it
within 1e-4, and GOF within the mixed-precision bound.  Shapes: one 128-node
block, several blocks (200 and 1,000 nodes), a static window longer than one
256-volume chunk, and the intra-hemisphere pair order."""
import numpy as np
import pytest

import cases
from cubnm_b200 import core, utils

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nodes,N,dur,ws,step,remove,exc", [(100, 24, 60, 10, 2, 30, False), (200, 8, 40, 8, 2, 4, False),
                                                            (68, 6, 320, 10, 20, 10, False), (100, 6, 40, 8, 2, 4, True),
                                                            (1000, 2, 12, 2, 1, 2, False)])
def test_tensor_core_fc_matches_fp64_fc(nodes, N, dur, ws, step, remove, exc):
    args = list(cases.synthetic_args("rWW", N=N, nodes=nodes, duration_s=dur, seed=nodes, density=0.2,
                                     precision="fp32", window_size=ws, window_step=step, bold_remove_s=remove))
    args[7] = dict(args[7], exc_interhemispheric=str(int(exc)))
    ref = core.run_simulations(*[a.copy() if isinstance(a, np.ndarray) else a for a in args])
    args[7] = dict(args[7], fc="tc")
    tc = core.run_simulations(*args)
    np.testing.assert_array_equal(tc["sim_bold"], ref["sim_bold"])   # the same integration
    assert np.abs(tc["sim_fc_trils"] - ref["sim_fc_trils"]).max() < 1e-4
    assert np.abs(tc["sim_fcd_trils"] - ref["sim_fcd_trils"]).max() < 1e-4
    emp = cases.synthetic_emp_bold(nodes, dur, 5)
    efc = utils.calculate_fc(emp, exc_interhemispheric=exc)
    g1 = utils.gof(ref["sim_fc_trils"], efc)
    g2 = utils.gof(tc["sim_fc_trils"], efc)
    for k in g1:
        assert np.abs(g1[k] - g2[k]).max() < 1e-3, k
