#!/usr/bin/env python
"""Cuts the reference's level-step kernels and its query planner out of its
HnGPU.cu, where the file lies, into build-only include files.

The reference's HnGPU.cu cannot be compiled for sm_100a as a whole: its level
driver ``hnSolve`` / ``hnLoop`` and ``hnScan`` (HnGPU.cu:336-669) launch
kernels and call ``cudaDeviceSynchronize`` and CUB from device code (CUDA
dynamic parallelism of the CDP1 kind, which sm_90 and later do not have).
Everything else it holds compiles unchanged.  This script writes, into the
output directory (git-ignored; never committed):

  hngpu_kernels.inc  HnGPU.cu from its first line up to the comment opening
                     hnScan -- cudaExit, reqExists, getBlockCount,
                     updateHeader and the kernels hnInit, hnGen, hnCheck,
                     hnRem, hnDeg, hnRemove (HnGPU.cu:1-334) -- and the
                     namespace's closing brace;
  hngpu_plan.inc     HnSetup::preProcessQuery (HnGPU.cu:749-816) inside its
                     namespace.

Nothing is edited: the text between the markers is copied byte for byte,
and the markers must occur exactly once, so a different reference version
fails loudly instead of building something else.

    python baseline/extract_ref.py <reference dir> <output dir>
"""
import os
import sys


def cut(text, start_marker, end_marker, include_end):
    a = text.count(start_marker)
    b = text.count(end_marker)
    if a != 1 or b < 1:
        raise SystemExit(f"marker not found exactly once: {start_marker!r} ({a}) / {end_marker!r} ({b})")
    i = text.index(start_marker)
    j = text.index(end_marker, i)
    return text[i:j + (len(end_marker) if include_end else 0)]


def main():
    ref, out = sys.argv[1], sys.argv[2]
    src = open(os.path.join(ref, "HnGPU.cu")).read()
    os.makedirs(out, exist_ok=True)
    # kernels: from the top of the file to the comment that opens hnScan
    scan_comment = "    /*\n    * Calls CUB implementation of Device-Wide Exclusive Scan"
    if src.count(scan_comment) != 1:
        raise SystemExit("hnScan marker not found exactly once")
    kernels = src[:src.index(scan_comment)]
    if kernels.count("namespace HnGPU {") != 1 or "hnRemove" not in kernels or "hnSolve" in kernels:
        raise SystemExit("unexpected kernel section")
    with open(os.path.join(out, "hngpu_kernels.inc"), "w") as f:
        f.write("// Generated from the reference's HnGPU.cu by baseline/extract_ref.py.\n")
        f.write(kernels)
        f.write("}  // namespace HnGPU\n")
    # planner: preProcessQuery, up to its return and closing brace
    plan = cut(src, "    __host__ uint32_t preProcessQuery(CCSR::CCSRGraph query",
               "        return maxValency;\n    }\n", True)
    with open(os.path.join(out, "hngpu_plan.inc"), "w") as f:
        f.write("// Generated from the reference's HnGPU.cu by baseline/extract_ref.py.\n")
        f.write("namespace HnSetup {\n")
        f.write(plan)
        f.write("}  // namespace HnSetup\n")
    print(f"wrote {out}/hngpu_kernels.inc ({kernels.count(chr(10))} lines), hngpu_plan.inc")


if __name__ == "__main__":
    main()
