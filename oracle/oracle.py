"""Python entry to the CPU oracle (test infrastructure only).

Loads ``oracle/liboracle.so`` (built by ``oracle/Makefile``) and exposes the
reference's ``cubnm.core`` calling convention on it, so tests can run the same
arguments through the oracle and through the product library and compare.
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it.
"""
import ctypes as C
import os
import subprocess

from cubnm_b200 import _abi

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def build():
    subprocess.run(["make", "-C", _HERE, "-s"], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        _LIB = C.CDLL(path)
        _abi.declare(_LIB, "oracle_")
        _LIB.oracle_num_threads.restype = C.c_int
        _LIB.oracle_init()
    return _LIB


def run_simulations(*args):
    """Same 22 positional arguments and output dict as cubnm.core.run_simulations."""
    return _abi.run(lib(), "oracle_", *args)


def init():
    lib().oracle_init()


def set_const(key, value):
    lib().oracle_set_const(key.encode(), float(value))


def num_threads():
    return lib().oracle_num_threads()
