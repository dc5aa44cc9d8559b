"""Test infrastructure: a CBMState stand-in built by the CPU oracle.

OracleState.new(con_text, act_text, n_zones, wiring_seeds) restates the
reference's CBMState(actPF, conPF, nZones, ...) initial values and
microzone wiring in the oracle (oracle/libcbm_oracle.so, cbm_oracle_new),
with the input-net tables left for the caller, and exposes the con() /
array() / writeState() calls that
cerebellum_simulation_b200.networks.build_random_network uses.  It lets the
CPU baseline of the benchmark build the same random network as the product
without loading the product's library.  Only tests and the benchmark's CPU
leg use it.
"""
import ctypes
import os
import subprocess

import numpy as np

ORACLE_DIR = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(ORACLE_DIR, "libcbm_oracle.so")

_lib = None


def _oracle():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_LIB):
            subprocess.run(["make", "-C", ORACLE_DIR, "oracle"], check=True, capture_output=True)
        lib = ctypes.CDLL(ORACLE_LIB)
        P, S, U32 = ctypes.c_void_p, ctypes.c_char_p, ctypes.c_uint32
        lib.cbm_oracle_new.restype = P
        lib.cbm_oracle_new.argtypes = [S, S, U32, P, ctypes.c_char_p, ctypes.c_size_t]
        lib.cbm_oracle_array.restype = P
        lib.cbm_oracle_array.argtypes = [P, S, ctypes.c_int, ctypes.POINTER(ctypes.c_uint64)]
        lib.cbm_oracle_con.restype = ctypes.c_int
        lib.cbm_oracle_con.argtypes = [P, S, ctypes.POINTER(U32)]
        lib.cbm_oracle_save.restype = ctypes.c_int
        lib.cbm_oracle_save.argtypes = [P, S]
        lib.cbm_oracle_free.argtypes = [P]
        _lib = lib
    return _lib


def _dtype(name):
    """Element type of a connectivity array by the reference's naming."""
    if name.startswith("nump"):
        return np.int32
    if name.startswith("has"):
        return np.uint8
    if name.startswith("p"):
        return np.uint32
    raise KeyError(f"no element type known for {name}")


class OracleState:
    def __init__(self, handle):
        self._h = handle

    @classmethod
    def new(cls, con_text, act_text, n_zones=1, wiring_seeds=None):
        lib = _oracle()
        seeds = None if wiring_seeds is None else np.ascontiguousarray(wiring_seeds, dtype=np.int32)
        err = ctypes.create_string_buffer(256)
        h = lib.cbm_oracle_new(con_text.encode(), act_text.encode(), n_zones,
                               None if seeds is None else seeds.ctypes.data, err, 256)
        if not h:
            raise ValueError(err.value.decode())
        st = cls(h)
        st._seeds = seeds
        return st

    def __del__(self):
        if getattr(self, "_h", None):
            _oracle().cbm_oracle_free(self._h)
            self._h = None

    def con(self, key):
        v = ctypes.c_uint32()
        if _oracle().cbm_oracle_con(self._h, key.encode(), ctypes.byref(v)):
            raise KeyError(key)
        return v.value

    def array(self, name, zone=-1):
        """numpy view of a connectivity array; writes go into the state."""
        n = ctypes.c_uint64()
        p = _oracle().cbm_oracle_array(self._h, name.encode(), zone, ctypes.byref(n))
        if not p:
            raise KeyError(name)
        dt = np.dtype(_dtype(name))
        buf = (ctypes.c_uint8 * n.value).from_address(p)
        buf._owner = self  # the view keeps the state alive
        return np.frombuffer(buf, dtype=dt)

    def writeState(self, path):
        if _oracle().cbm_oracle_save(self._h, os.fsencode(path)):
            raise OSError(f"cannot write {path}")
