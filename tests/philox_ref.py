"""Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as
1, 2, 3", SC 2011) restated in numpy, with the Box-Muller transform the library's
"philox" noise mode applies (test infrastructure)."""
import numpy as np

M0, M1 = np.uint64(0xD2511F53), np.uint64(0xCD9E8D57)
W0, W1 = np.uint32(0x9E3779B9), np.uint32(0xBB67AE85)
MASK = np.uint64(0xFFFFFFFF)


def philox4x32_10(ctr, key):
    """ctr: uint32 [..., 4]; key: uint32 [2] -> uint32 [..., 4]."""
    c = [np.asarray(ctr[..., i], dtype=np.uint64) for i in range(4)]
    k0, k1 = np.uint64(key[0]), np.uint64(key[1])
    for r in range(10):
        p0 = M0 * c[0]
        p1 = M1 * c[2]
        hi0, lo0 = p0 >> np.uint64(32), p0 & MASK
        hi1, lo1 = p1 >> np.uint64(32), p1 & MASK
        c = [hi1 ^ c[1] ^ k0, lo1, hi0 ^ c[3] ^ k1, lo0]
        k0 = (k0 + np.uint64(W0)) & MASK
        k1 = (k1 + np.uint64(W1)) & MASK
    return np.stack([x.astype(np.uint32) for x in c], axis=-1)


def philox_normals(seed, count):
    """The noise array of the "philox" mode: counter i = (i, 0, 0, 0), key = (seed, 0);
    the four words give two 53-bit uniforms u1 = ((w0 << 32 | w1) >> 11 + 1/2) 2^-53,
    u2 likewise from (w2, w3), and z = sqrt(-2 ln u1) (cos 2 pi u2, sin 2 pi u2)."""
    n_ctr = (count + 1) // 2
    ctr = np.zeros((n_ctr, 4), dtype=np.uint32)
    ctr[:, 0] = np.arange(n_ctr, dtype=np.uint64).astype(np.uint32)
    w = philox4x32_10(ctr, np.array([seed & 0xFFFFFFFF, 0], dtype=np.uint32)).astype(np.uint64)
    a = ((w[:, 0] << np.uint64(32)) | w[:, 1]) >> np.uint64(11)
    b = ((w[:, 2] << np.uint64(32)) | w[:, 3]) >> np.uint64(11)
    u1 = (a.astype(np.float64) + 0.5) * 2.0 ** -53
    u2 = (b.astype(np.float64) + 0.5) * 2.0 ** -53
    r = np.sqrt(-2.0 * np.log(u1))
    z = np.empty(2 * n_ctr)
    z[0::2] = r * np.cos(2 * np.pi * u2)
    z[1::2] = r * np.sin(2 * np.pi * u2)
    return z[:count]
