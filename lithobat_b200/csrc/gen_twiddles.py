"""Write twiddles.cuh: the 64th roots of unity as FP32 literals.

cos/sin(2*pi*k/64) are evaluated in FP64 by the host's libm and printed with
17 significant digits, so the compiler's decimal-to-float conversion gives
the correctly rounded FP32 value. Run by the build step.
"""
import math
import sys
from pathlib import Path


def main(out: Path) -> None:
    lines = [
        "// Generated by gen_twiddles.py. exp(2*pi*i*k/64) for k = 0..63.",
        "#pragma once",
        "namespace litho {",
        "__device__ __forceinline__ float tw64_re(int k) {",
        "  switch (k & 63) {",
    ]
    for k in range(64):
        lines.append(f"    case {k}: return {math.cos(2 * math.pi * k / 64):.17e}f;")
    lines += ["  }", "  return 0.f;", "}", "__device__ __forceinline__ float tw64_im(int k) {",
              "  switch (k & 63) {"]
    for k in range(64):
        lines.append(f"    case {k}: return {math.sin(2 * math.pi * k / 64):.17e}f;")
    lines += ["  }", "  return 0.f;", "}", "}  // namespace litho", ""]
    out.write_text("\n".join(lines))


if __name__ == "__main__":
    main(Path(sys.argv[1]) if len(sys.argv) > 1 else Path(__file__).with_name("twiddles.cuh"))
