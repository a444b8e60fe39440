"""glibc-order powf: exp2 table derivation and agreement with the reference."""

import re
import struct
from decimal import Decimal, getcontext
from pathlib import Path

import numpy as np

from fixtures import inputs, load_golden
from oracle.powf import EXP2_TABLE, powf_gnu

HEADER = Path(__file__).resolve().parent.parent / "gpuwm-hex_b200" / "csrc" / "powf_gnu.cuh"


def derived_table():
    getcontext().prec = 60
    out = []
    for i in range(32):
        d = float(Decimal(2) ** (Decimal(i) / Decimal(32)))
        bits = struct.unpack("<Q", struct.pack("<d", d))[0]
        out.append((bits - (i << 47)) % (1 << 64))
    return out


def test_exp2_table_is_its_definition():
    table = derived_table()
    assert [int(x) for x in EXP2_TABLE] == table
    text = HEADER.read_text()
    macro = text[text.index("#define HEXDYN_EXP2_TABLE"):text.index("static __device__ __constant__ uint64_t")]
    device = [int(h, 16) for h in re.findall(r"0x([0-9a-f]{16})ull", macro)]
    assert device == table


def test_exner_of_rebuilt_sidecar_matches_reference():
    """The reference's first-step Exner is its powf of the t0 state; the
    carried sidecar after the step holds the recovered Exner (stage 3)."""
    fx = load_golden("l2_L12")
    arr = inputs(fx)
    zz = arr["vertical.zz"]
    rt = fx["dry.step1.rho_theta"]
    ex = powf_gnu((zz * np.float32(287.0 / 100000.0)) * rt, np.float32(287.0 / (1004.5 - 287.0)))
    assert np.array_equal(ex.view(np.uint32), fx["dry.step1.side.exner"].view(np.uint32))


def test_powf_close_to_libm():
    x = np.random.default_rng(0).uniform(0.05, 3.0, 100000).astype(np.float32)
    y = np.float32(287.0 / 717.5)
    ours = powf_gnu(x, y).astype(np.float64)
    exact = np.power(x.astype(np.float64), float(y))
    ulp = np.spacing(exact.astype(np.float32)).astype(np.float64)
    assert np.max(np.abs(ours - exact) / ulp) < 1.0
