#!/usr/bin/env python3
"""Writes csrc/dft_consts.cuh: cos/sin(2 pi m / R) for the odd prime DFT
lengths R in {3, 5, 11, 31}, evaluated in double precision and rounded once
to binary32; each table also as (v, v) float2 pairs, the operand form of the
packed FP32 instructions (__ffma2_rn) that apply one constant to the real and
imaginary parts of a complex value at once."""
import math
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def fmt(v):
    return "%.9ef" % float(np.float32(v))


def main():
    out = ["// Generated constants: cos/sin(2*pi*m/R) rounded to float, R in {3,5,11,31}.",
           "// Produced by evaluating the trigonometric functions in double precision (Python math) and",
           "// rounding once to binary32 (tart-gnss_b200/gen_dft_consts.py).  The *x2 tables hold each value",
           "// twice, as the (re, im) operand of packed FP32 instructions.",
           "#pragma once", ""]
    for R in (3, 5, 11, 31):
        c = [math.cos(2 * math.pi * m / R) for m in range(R)]
        s = [math.sin(2 * math.pi * m / R) for m in range(R)]
        out.append("__constant__ float kCos%d[%d] = {%s};" % (R, R, ", ".join(fmt(v) for v in c)))
        out.append("__constant__ float kSin%d[%d] = {%s};" % (R, R, ", ".join(fmt(v) for v in s)))
        out.append("__constant__ float2 kCos%dx2[%d] = {%s};" % (R, R, ", ".join("{%s, %s}" % (fmt(v), fmt(v)) for v in c)))
        out.append("__constant__ float2 kSin%dx2[%d] = {%s};" % (R, R, ", ".join("{%s, %s}" % (fmt(v), fmt(v)) for v in s)))
    open(os.path.join(HERE, "csrc", "dft_consts.cuh"), "w").write("\n".join(out) + "\n")


if __name__ == "__main__":
    main()
