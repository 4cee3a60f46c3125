"""cubnm_b200: B200-native simulation path for cuBNM-style brain network models.

``cubnm_b200.core`` is a drop-in for the reference's ``cubnm.core`` extension
(run_simulations / init / set_const); ``cubnm_b200.sim`` holds SimGroup classes
with the reference's run / score interface; ``cubnm_b200.utils`` the empirical
FC/FCD helpers and the GPU goodness-of-fit functions.
"""
__version__ = "0.1.0"
