"""The numpy Philox4x32-10 restatement against the published known-answer
vectors of the Random123 distribution (Salmon et al., SC 2011), and the
distribution of its Box-Muller normals (CPU)."""
import numpy as np
import scipy.stats

import philox_ref as P

KAT = [((0, 0, 0, 0), (0, 0), (0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8)),
       ((0xffffffff,) * 4, (0xffffffff, 0xffffffff), (0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd)),
       ((0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344), (0xa4093822, 0x299f31d0),
        (0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1))]


def test_philox_known_answers():
    for ctr, key, expect in KAT:
        got = P.philox4x32_10(np.array(ctr, dtype=np.uint32)[None], np.array(key, dtype=np.uint32))[0]
        assert [int(x) for x in got] == list(expect)


def test_philox_normals_are_standard_normal():
    z = P.philox_normals(7, 400001)
    assert z.shape == (400001,)
    assert abs(z.mean()) < 5e-3 and abs(z.var() - 1) < 1e-2
    assert scipy.stats.kstest(z[:20000], "norm").pvalue > 1e-3
    assert abs(np.corrcoef(z[:-1], z[1:])[0, 1]) < 5e-3
