"""Oracle (test infrastructure only): glibc-order single-precision powf.

The Exner function of the dycore is ``powf(zz*R/p0*rho_theta, R/(cp-R))`` in
the order of GNU libc 2.39 ``powf`` (``hexcore/native_powf.py:18``
``powf_native_gnu``), which is the published algorithm of Arm
optimized-routines v21.02 ``math/powf.c`` (MIT licence, Copyright (c)
2017-2019 Arm Limited): log2 through a 16-entry table of (1/c, log2 c) and a
degree-5 polynomial, then exp2 through a 32-entry table of 2^(i/32) and a
cubic, all in double precision with no fused multiply-adds, rounded to
binary32 at the end.

The log table and polynomial coefficients are Arm's published data and must
equal them bit for bit for the result to; the exp2 table is derived here from
its definition (bits of 2^(i/32) minus i<<47).  Only positive normal inputs
are admitted (the dycore's Exner argument is always one); anything else
raises instead of silently taking another path.
"""

from __future__ import annotations

import struct
from decimal import Decimal, getcontext

import numpy as np

_H = float.fromhex

# (1/c, log2 c) for the 16 subintervals of [0x3f330000, 2*0x3f330000).
LOG2_TABLE = np.array([
    (_H("0x1.661ec79f8f3bep+0"), _H("-0x1.efec65b963019p-2")),
    (_H("0x1.571ed4aaf883dp+0"), _H("-0x1.b0b6832d4fca4p-2")),
    (_H("0x1.49539f0f010bp+0"), _H("-0x1.7418b0a1fb77bp-2")),
    (_H("0x1.3c995b0b80385p+0"), _H("-0x1.39de91a6dcf7bp-2")),
    (_H("0x1.30d190c8864a5p+0"), _H("-0x1.01d9bf3f2b631p-2")),
    (_H("0x1.25e227b0b8eap+0"), _H("-0x1.97c1d1b3b7afp-3")),
    (_H("0x1.1bb4a4a1a343fp+0"), _H("-0x1.2f9e393af3c9fp-3")),
    (_H("0x1.12358f08ae5bap+0"), _H("-0x1.960cbbf788d5cp-4")),
    (_H("0x1.0953f419900a7p+0"), _H("-0x1.a6f9db6475fcep-5")),
    (_H("0x1p+0"), 0.0),
    (_H("0x1.e608cfd9a47acp-1"), _H("0x1.338ca9f24f53dp-4")),
    (_H("0x1.ca4b31f026aap-1"), _H("0x1.476a9543891bap-3")),
    (_H("0x1.b2036576afce6p-1"), _H("0x1.e840b4ac4e4d2p-3")),
    (_H("0x1.9c2d163a1aa2dp-1"), _H("0x1.40645f0c6651cp-2")),
    (_H("0x1.886e6037841edp-1"), _H("0x1.88e9c2c1b9ff8p-2")),
    (_H("0x1.767dcf5534862p-1"), _H("0x1.ce0a44eb17bccp-2")),
], dtype=np.float64)

LOG2_POLY = np.array([
    _H("0x1.27616c9496e0bp-2"), _H("-0x1.71969a075c67ap-2"),
    _H("0x1.ec70a6ca7baddp-2"), _H("-0x1.7154748bef6c8p-1"),
    _H("0x1.71547652ab82bp0"),
], dtype=np.float64)

EXP2_POLY = (_H("0x1.c6af84b912394p-5"), _H("0x1.ebfce50fac4f3p-3"),
             _H("0x1.62e42ff0c52d6p-1"))
EXP2_SHIFT = _H("0x1.8p+47")


def _exp2_table() -> np.ndarray:
    getcontext().prec = 60
    out = np.empty(32, dtype=np.uint64)
    for i in range(32):
        d = float(Decimal(2) ** (Decimal(i) / Decimal(32)))
        bits = struct.unpack("<Q", struct.pack("<d", d))[0]
        out[i] = (bits - (i << 47)) % (1 << 64)
    return out


EXP2_TABLE = _exp2_table()


def powf_gnu(base: np.ndarray, exponent: np.float32) -> np.ndarray:
    """``powf(base, exponent)`` for positive normal FP32 ``base``."""
    x = np.ascontiguousarray(base, dtype=np.float32)
    ix = x.reshape(-1).view(np.uint32)
    if not np.all((ix >= 0x00800000) & (ix < 0x7F800000)):
        raise FloatingPointError("powf oracle admits only positive normal bases")
    tmp = ix - np.uint32(0x3F330000)
    index = (tmp >> np.uint32(19)) % 16
    top = tmp & np.uint32(0xFF800000)
    z = (ix - top).view(np.float32).astype(np.float64)
    k = (top.view(np.int32) >> 23).astype(np.float64)
    invc, logc = LOG2_TABLE[index, 0], LOG2_TABLE[index, 1]
    r = z * invc - 1.0
    y0 = logc + k
    r2 = r * r
    r4 = r2 * r2
    a = LOG2_POLY
    y = a[0] * r + a[1]
    p = a[2] * r + a[3]
    q = a[4] * r + y0
    q = p * r2 + q
    y = y * r4 + q
    xd = np.float64(np.float32(exponent)) * y
    if np.any(np.abs(xd) > 1000.0):
        raise FloatingPointError("powf oracle: exponent range outside the dycore's")
    kd = xd + EXP2_SHIFT
    ki = kd.view(np.uint64)
    r = xd - (kd - EXP2_SHIFT)
    t = EXP2_TABLE[ki % np.uint64(32)] + (ki << np.uint64(47))
    scale = t.view(np.float64)
    c0, c1, c2 = EXP2_POLY
    zz = c0 * r + c1
    r2 = r * r
    yy = c2 * r + 1.0
    yy = zz * r2 + yy
    return (yy * scale).astype(np.float32).reshape(x.shape)
